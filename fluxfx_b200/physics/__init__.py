"""Descriptors and small host-side helpers of the smoke step (no device code)."""
