"""Utilities kept from the reference (src/utilites.py:18-24)."""
from __future__ import annotations

__all__ = ["get_index"]


def get_index(N, n, rank):
    """Slab bounds of ``rank`` among ``n`` ranks (remainder to the first ranks)."""
    batch_size = N // n
    remaining = N % n
    if rank < remaining:
        return (rank * (batch_size + 1), (rank + 1) * (batch_size + 1))
    return (rank * batch_size + remaining, (rank + 1) * batch_size + remaining)
