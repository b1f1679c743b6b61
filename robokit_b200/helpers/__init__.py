"""Helpers over the LM-IK path (robokit helpers/)."""
