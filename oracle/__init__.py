"""Parity oracle for the dmsc_b200 CUDA path (test infrastructure only)."""
