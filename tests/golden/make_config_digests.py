"""Generates tests/golden/config_<name>.npz: the final-state digests of the
four benchmark configurations at their stated sizes, from the compiled
reference core (oracle/_ref), for tests/test_configs_gpu.py.

Run where the oracle libraries are built (one configuration per process; the
collapse case holds about 30 GB of reference block storage and runs for
hours on one core):
    python tests/golden/make_config_digests.py sod1024
    python tests/golden/make_config_digests.py fourier128
    python tests/golden/make_config_digests.py blast_root8
    python tests/golden/make_config_digests.py collapse_root12 [--steps N]

The reference runs its own driver loop (rh_run: src/main.c:485-562) from the
oracle's initial state; the digests are taken over every active block (see
tests/config_cases.py).  --steps lowers the step count (the GPU test runs
whatever step count the fixture records).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as R  # noqa: E402
from tests import config_cases as CC  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CC.CASES))
    ap.add_argument("--steps", type=int, default=0)
    args = ap.parse_args()
    case = CC.CASES[args.case]
    steps = args.steps or case.steps
    ref = R.Reference(case.mhd)
    p = case.params()
    t0 = time.time()
    ref.setup(p)
    t_setup = time.time() - t0
    ints, _, _ = ref.mesh_arrays()
    active = np.nonzero(ints[:, 2] == 1)[0]
    levels = np.bincount(ints[active, 1]).tolist()
    print(f"{args.case}: {ref.nblocks()} blocks, {len(active)} active, per level {levels}, "
          f"set-up {t_setup:.1f} s", flush=True)
    t0 = time.time()
    done = 0
    chunk = 10
    st = None
    while done < steps:
        n, t, dt, step = ref.run(min(chunk, steps - done))
        st = (t, dt, step)
        done += n
        print(f"  step {step}: t = {t:.6e}, dt = {dt:.6e}, {time.time() - t0:.0f} s", flush=True)
        if n == 0 or t >= p.t_end:
            break
    secs = time.time() - t0
    md = CC.MeshDigest(active, ref.nhydro, R.NCELLS, R.NFACES, case.mhd)
    for b in active:
        md.add(b, ref.W(b), [ref.Bf(b, d) for d in range(3)] if case.mhd else None)
    out = md.arrays()
    out.update({
        "t": np.float64(st[0]), "dt": np.float64(st[1]), "step": np.int64(st[2]),
        "steps_requested": np.int64(steps), "levels": np.asarray(levels),
        "nblocks": np.int64(ref.nblocks()), "ref_seconds": np.float64(secs),
    })
    path = os.path.join(HERE, f"config_{args.case}.npz")
    np.savez_compressed(path, **out)
    print(f"{args.case}: {st[2]} steps, t = {st[0]!r}, {secs:.0f} s of reference time "
          f"({len(active) * 4096 * st[2] / secs:.3e} zone-updates/s, one core) -> {path}", flush=True)


if __name__ == "__main__":
    main()
