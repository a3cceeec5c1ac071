"""group::Group (src/group.rs:11-69)."""
from __future__ import annotations

import enum


class Group(enum.IntEnum):
    G1 = 1  # coordinates in Fq
    G2 = 2  # coordinates in Fq2 = Fq[u]/(u^2 + 1)

    def affine_words(self) -> int:
        """u32 words of one affine point (x then y; Fq2 as a then b)."""
        return 16 if self is Group.G1 else 32

    def xyzz_words(self) -> int:
        """u32 words of one XYZZ accumulator point."""
        return 2 * self.affine_words()
