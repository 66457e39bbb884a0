"""Oracle package: CPU checker for the CUDA path (test infrastructure only)."""
