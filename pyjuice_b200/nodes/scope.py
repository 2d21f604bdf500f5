"""Variable scopes of circuit nodes.

A scope is a set of variable ids stored as a Python integer bitmask. It offers the
operations the compiler and the structure builders use on the reference's
``pyjuice.utils.BitSet`` (src/pyjuice/utils/bitset.py:6): ``from_array``,
``to_list`` (ascending ids), ``&``, ``|``, ``len``, equality and hashing.
"""

from __future__ import annotations

from typing import Iterable


class BitSet:
    __slots__ = ("_bits",)

    def __init__(self, bits: int = 0):
        self._bits = int(bits)

    @classmethod
    def from_array(cls, arr: Iterable[int]) -> "BitSet":
        bits = 0
        for v in arr:
            v = int(v)
            if v < 0:
                raise ValueError(f"variable ids must be non-negative, got {v}")
            bits |= 1 << v
        return cls(bits)

    def to_list(self):
        out = []
        bits = self._bits
        v = 0
        while bits:
            if bits & 1:
                out.append(v)
            bits >>= 1
            v += 1
        return out

    def add(self, v: int):
        self._bits |= 1 << int(v)

    def hasitem(self, v: int) -> bool:
        return (self._bits >> int(v)) & 1 == 1

    def __contains__(self, v):
        return self.hasitem(v)

    def __and__(self, other: "BitSet") -> "BitSet":
        return BitSet(self._bits & other._bits)

    def __or__(self, other: "BitSet") -> "BitSet":
        return BitSet(self._bits | other._bits)

    def __ior__(self, other: "BitSet") -> "BitSet":
        self._bits |= other._bits
        return self

    def __len__(self) -> int:
        return bin(self._bits).count("1")

    def __iter__(self):
        return iter(self.to_list())

    def __eq__(self, other) -> bool:
        return isinstance(other, BitSet) and self._bits == other._bits

    def __hash__(self) -> int:
        return hash(("BitSet", self._bits))

    def __repr__(self) -> str:
        return f"BitSet({self.to_list()})"

    def contains_all(self, other: "BitSet") -> bool:
        return (self._bits & other._bits) == other._bits

    def contains_any(self, other: "BitSet") -> bool:
        return (self._bits & other._bits) != 0
