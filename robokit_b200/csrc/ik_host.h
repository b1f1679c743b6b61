// ik_host.h — host-side pieces of libb200ik shared by its translation units:
// the host copy of a robot, lowered terms, the table-blob builder and launch
// helpers.  Internal; the public interface is include/b200ik.h.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "b200ik.h"
#include "ik_tables.h"

namespace b200ik {
namespace host {

// Host copy of a robot with the derived tables the kernels read.
struct RobotHost {
    int nj = 0, nl = 0, na = 0, ns = 0;
    std::vector<int> jtype, jparent, jact, jmimic, lpj, sphlink;
    std::vector<float> jmul, joff, jaxis, jpt, lim, sph, lbound;
    std::vector<unsigned long long> lanc;  // per link: ancestor joints
    std::vector<int> jorder;               // joints in topological order
    std::vector<int> colstart, coljoint;
    std::vector<float> colmul;
    int fk_rounds = 0;
};

}  // namespace host
}  // namespace b200ik

// A robot registered with ik_robot_create: its host copy and the robot-only
// table blobs (fixed base / floating base) used by the FK and Jacobian stages.
struct IkRobot {
    b200ik::host::RobotHost h;
    char* d_blob[2] = {nullptr, nullptr};
    int blob_bytes[2] = {0, 0};
    int ws_bytes[2] = {0, 0};
};

namespace b200ik {
namespace host {

// One validated term descriptor with host copies of its arrays.
struct TermHost {
    IkTermDesc d;
    std::vector<int> frame_links;
    std::vector<float> weights;
    std::vector<float> vlim;  // velocity-limit terms: [na]
    std::vector<int> qsph;      // scene collision: queried sphere indices
    std::vector<float> selem;   // scene collision: primitive records (5 float4 each), sorted by scene
    std::vector<int> soff;      // scene collision: CSR offsets per scene
    std::vector<int> lp, lpoff, sp;
    int row = 0, rows = 0;
};

// The lowered problem: table blob + sizes.
struct ProblemTables {
    std::vector<char> blob;
    int blob_bytes = 0, ws_bytes = 0, D = 0, R = 0, E = 0;
};

int fail(int code, const char* fmt, ...);
int num_sms();
int max_smem_optin();
int smem_bytes(int blob_bytes, int ws_bytes, int G);
int choose_group(int D, int blob_bytes, int ws_bytes, int requested);
int check_params(const IkLmParams* p);
int check_launch();

// Validate a robot descriptor and build its host copy.
int fill_robot(const IkRobotDesc* d, RobotHost& r);
// Validate terms against a robot and copy them; R = rows in the reference layout.
int fill_terms(const RobotHost& r, int floating, const IkTermDesc* terms, int num_terms, std::vector<TermHost>& out,
               int& R);
// Lower robot + terms + active-DOF mask (empty = none) into the table blob.
int build_tables(const RobotHost& r, int floating, const std::vector<TermHost>& terms, const std::vector<float>& mask,
                 int R, ProblemTables& out);

template <typename K>
int prepare_kernel(K kernel, int smem) {
    if (smem > max_smem_optin()) return fail(IK_E_UNSUPPORTED, "shared memory %d B exceeds the device limit", smem);
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return fail(IK_E_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    return IK_OK;
}

template <typename K>
int grid_for(K kernel, int smem, int batch, int G, int blocks_per_sm_req, int& grid, int block_threads) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block_threads, smem);
    if (e != cudaSuccess) return fail(IK_E_CUDA, "occupancy query: %s", cudaGetErrorString(e));
    if (per_sm <= 0) return fail(IK_E_UNSUPPORTED, "kernel does not fit on an SM (smem %d B)", smem);
    if (blocks_per_sm_req > 0 && blocks_per_sm_req < per_sm) per_sm = blocks_per_sm_req;
    const int gpb = block_threads / G;
    const int need = (batch + gpb - 1) / gpb;
    grid = need < per_sm * num_sms() ? need : per_sm * num_sms();
    if (grid < 1) grid = 1;
    return IK_OK;
}

}  // namespace host
}  // namespace b200ik
