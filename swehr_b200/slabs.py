"""Row-slab decomposition of one domain over ranks (host-side plan).

A domain too large for one GPU, or one that should finish sooner, splits
along i into slabs of whole rows, one per rank.  A step of SWEHR reads, for
row i, the previous state of rows i-1..i+1 (face fluxes, the density
gradient, the deposit neighbours of the slope-failure test) and the
topography of rows i-2..i+2 (the central slopes of the neighbours whose
stale or fresh SLOPEX the failure test reads, SWEHR.c:1293, and the lagged
GZ of the lower face's left cell, SWEHR.c:1135), so each slab carries
HALO = 2 rows of its neighbours on each inner side, refreshed before every
step, and the time step needs one scalar reduction per step: the largest
wave speed over all faces (SWEHR.c:1408).  A face belongs to the slab that
owns its lower (left) row, face 1/2 to the first slab, so every face is
counted once.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Tuple

HALO = 2


@dataclass(frozen=True)
class Slab:
    rank: int
    own: Tuple[int, int]        # global rows a..b (1-based, inclusive) this rank owns
    span: Tuple[int, int]       # global rows held: own plus up to HALO neighbour rows each side

    @property
    def local_own(self) -> Tuple[int, int]:
        """the owned rows in the slab's local numbering (1-based)"""
        return self.own[0] - self.span[0] + 1, self.own[1] - self.span[0] + 1

    @property
    def rows(self) -> int:
        return self.span[1] - self.span[0] + 1


def plan(nx: int, world: int, halo: int = HALO) -> List[Slab]:
    """Split rows 1..nx into `world` slabs of nearly equal height (the first
    nx % world slabs one row taller), each with its halo span."""
    if world < 1 or nx < world * halo:
        raise ValueError("need 1 <= world and at least `halo` rows per slab")
    base, extra = divmod(nx, world)
    out, a = [], 1
    for r in range(world):
        b = a + base - 1 + (1 if r < extra else 0)
        out.append(Slab(r, (a, b), (max(1, a - halo), min(nx, b + halo))))
        a = b + 1
    return out


def exchanges(slabs: List[Slab], halo: int = HALO):
    """The halo refresh before a step as (src_rank, src_rows, dst_rank,
    dst_rows) in global rows: each slab's first/last `halo` owned rows go to
    the neighbour whose span holds them."""
    out = []
    for s, t in zip(slabs, slabs[1:]):
        up = (s.own[1] - halo + 1, s.own[1])            # s's top owned rows -> t's lower halo
        lo = (t.own[0], t.own[0] + halo - 1)            # t's bottom owned rows -> s's upper halo
        up = (max(up[0], s.own[0]), up[1])
        lo = (lo[0], min(lo[1], t.own[1]))
        out.append((s.rank, up, t.rank, up))
        out.append((t.rank, lo, s.rank, lo))
    return out
