"""Learned pressure warm start (U-Net on the library's BF16 tensor-core convolutions)."""
