"""Validation harnesses of the reference's experiments run on the GPU path."""
