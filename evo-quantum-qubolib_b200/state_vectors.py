"""Bit-packed state vectors (src/qubo_lib/state_vectors.py:6-79).

Packing convention, kept identical to the reference: bit j of a row goes to element
``j // bits`` at bit position ``j % bits`` (LSB first inside each element); the default
element type is uint8.
"""
from __future__ import annotations

import numpy as np


class StateVectors:
    SUPPORTED_TYPES = {np.uint8, np.uint16, np.uint32, np.uint64, np.int8, np.int16, np.int32, np.int64}

    def __init__(self, wide_vector_matrix: np.ndarray):
        wide = np.asarray(wide_vector_matrix)
        self.N = wide.shape[1]
        self.element_bits = 8
        self.bitwise_vectors = self.pack_wide_vectors_to_bitwise(wide)

    @classmethod
    def from_packed_vectors(cls, packed_vector_matrix: np.ndarray, N: int) -> "StateVectors":
        if packed_vector_matrix.dtype.type not in cls.SUPPORTED_TYPES:
            raise TypeError(f"Unsupported dtype: {packed_vector_matrix.dtype}. Supported types: {cls.SUPPORTED_TYPES}")
        inst = cls.__new__(cls)
        inst.bitwise_vectors = packed_vector_matrix
        inst.N = N
        inst.element_bits = packed_vector_matrix.dtype.itemsize * 8
        return inst

    def pack_wide_vectors_to_bitwise(self, wide_vectors: np.ndarray, target_dtype=np.uint8) -> np.ndarray:
        if target_dtype not in self.SUPPORTED_TYPES:
            raise TypeError(f"Unsupported target dtype: {target_dtype}. Supported types: {self.SUPPORTED_TYPES}")
        if target_dtype is np.uint8:  # the default: numpy's LSB-first byte packing is this layout
            return np.packbits(np.asarray(wide_vectors) != 0, axis=1, bitorder="little")
        rows, length = wide_vectors.shape
        bits = np.dtype(target_dtype).itemsize * 8
        per_row = (length + bits - 1) // bits
        nz = np.zeros((rows, per_row * bits), dtype=np.uint64)
        nz[:, :length] = (wide_vectors != 0)
        weights = (np.uint64(1) << np.arange(bits, dtype=np.uint64))
        packed = (nz.reshape(rows, per_row, bits) * weights).sum(axis=2, dtype=np.uint64)
        return packed.astype(target_dtype)

    def get_wide_vectors(self) -> np.ndarray:
        if self.bitwise_vectors is None:
            return np.array([])
        rows, _ = self.bitwise_vectors.shape
        j = np.arange(self.N)
        el = self.bitwise_vectors[:, j // self.element_bits].astype(np.uint64)
        return ((el >> (j % self.element_bits).astype(np.uint64)) & np.uint64(1)).astype(np.uint8).reshape(rows, self.N)
