"""The four benchmark configurations at their stated sizes, and the state
digests that pin them.

Each case runs the reference's driver loop (src/main.c:485-562: calc_dt, the
dt_factor growth limit, the t_end clip, the RK2 step, the dt_src clamp) for
the stated number of steps from the oracle's initial state.  The digests of
the final state are generated once from the compiled reference core by
tests/golden/make_config_digests.py and committed as small fixtures; the GPU
tests (tests/test_configs_gpu.py) run the same configuration from the same
initial state through the C ABI and compare.

Digest of one block: SHA-256 over its whole W array (every variable, both
stage slots, ghost cells included; the reference layout [var][slot][cell])
followed by its three Bf arrays (both slots, every face), as little-endian
doubles after x + 0.0, which maps -0.0 to +0.0 and leaves every other value
unchanged.  Equal digests therefore mean the arrays compare equal element by
element as doubles (the test of np.array_equal); a second, strict digest of
the raw bits of the whole mesh is kept beside it.  A seeded sample of active
cells and faces (slot 0) is stored too, so that a digest mismatch can still
be measured as a relative error.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

NSAMPLE = 2048


@dataclass(frozen=True)
class Case:
    name: str
    mhd: bool
    steps: int          # driver steps (an upper bound when the run ends at t_end)
    gravity: bool
    what: str

    def params(self):
        from oracle import ref as R
        if self.name == "sod1024":
            return R.params_sod(nblocks_x=64, t_end=0.2)
        if self.name == "fourier128":
            return R.params_fourier(root=8, nmodes=32, kmax=4)
        if self.name == "blast_root8":
            return R.params_amr_blast(root=8, max_level=2, radii=(0.4, 0.2))
        if self.name == "collapse_root12":
            return R.params_collapse(root=12)
        raise KeyError(self.name)


CASES = {
    c.name: c for c in (
        Case("sod1024", False, 100000, False,
             "Sod tube, 64 blocks of 16^3 along x (1024 cells), gamma 1.4, HLLC, run to t = 0.2"),
        Case("fourier128", True, 20, False,
             "Fourier-mode MHD, 128^3 = 512 blocks, 32 modes |k| <= 4, 20 RK2 steps"),
        Case("blast_root8", True, 50, False,
             "magnetised blast, 8^3 roots on [-0.7, 0.7]^3, 3 levels (r < 0.4 / 0.2), 50 RK2 steps"),
        Case("collapse_root12", True, 100, True,
             "gravity collapse, 12^3 roots on [-1, 1]^3, 4 levels (r < 0.4 / 0.2 / 0.1), 100 RK2 steps"),
    )
}


def _canon(a: np.ndarray) -> bytes:
    return (np.ascontiguousarray(a, dtype="<f8") + 0.0).tobytes()


def block_digest(W: np.ndarray, Bf) -> bytes:
    """W: the block's flat W array; Bf: its three Bf arrays (or None)."""
    h = hashlib.sha256()
    h.update(_canon(W))
    if Bf is not None:
        for d in range(3):
            h.update(_canon(Bf[d]))
    return h.digest()


class MeshDigest:
    """Accumulates per-block digests, the strict whole-mesh digest and the
    sample values, block by block (so no full copy of the mesh is needed)."""

    def __init__(self, active, nv, ncells, nfaces, mhd, seed=20261203):
        from tests import helpers as H
        self.active = np.asarray(active, dtype=np.int64)
        self.mhd = mhd
        self.nv = nv
        self.ncells = ncells
        rng = np.random.default_rng(seed)
        pos = rng.integers(0, len(self.active), NSAMPLE)
        self.cell_block = self.active[pos]
        self.cell = rng.choice(H.active_cells(), NSAMPLE)
        self.face_block = self.active[rng.integers(0, len(self.active), (3, NSAMPLE))]
        self.face = np.stack([rng.choice(H.active_faces(d), NSAMPLE) for d in range(3)])
        self.nfaces = nfaces
        self.digests = {}
        self.strict = hashlib.sha256()
        self.cell_vals = np.full((NSAMPLE, nv), np.nan)
        self.face_vals = np.full((3, NSAMPLE), np.nan)

    def add(self, b: int, W: np.ndarray, Bf) -> None:
        """Blocks must be added in the order of `active`."""
        self.digests[int(b)] = block_digest(W, Bf)
        self.strict.update(np.ascontiguousarray(W, dtype="<f8").tobytes())
        if Bf is not None:
            for d in range(3):
                self.strict.update(np.ascontiguousarray(Bf[d], dtype="<f8").tobytes())
        Wv = np.asarray(W).reshape(self.nv, -1, self.ncells)
        m = self.cell_block == b
        if m.any():
            self.cell_vals[m] = Wv[:, 0, self.cell[m]].T
        if Bf is not None:
            for d in range(3):
                m = self.face_block[d] == b
                if m.any():
                    self.face_vals[d, m] = np.asarray(Bf[d]).reshape(-1, self.nfaces)[0, self.face[d, m]]

    def block_digests(self) -> np.ndarray:
        return np.stack([np.frombuffer(self.digests[int(b)], dtype=np.uint8) for b in self.active])

    def arrays(self) -> dict:
        return {
            "active": self.active,
            "block_digests": self.block_digests(),
            "strict_digest": np.frombuffer(self.strict.digest(), dtype=np.uint8),
            "cell_block": self.cell_block, "cell": self.cell, "cell_vals": self.cell_vals,
            "face_block": self.face_block, "face": self.face, "face_vals": self.face_vals,
        }
