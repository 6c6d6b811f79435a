"""CPU checker for the CUDA path (test infrastructure only; never imported by the product)."""
