"""Readers of on-disk inputs (mirror of ebsdtorch/io/)."""

from .read_master_pattern import master_pattern_from_emsoft, read_master_pattern

__all__ = ["master_pattern_from_emsoft", "read_master_pattern"]
