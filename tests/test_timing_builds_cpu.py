"""The CPU baseline times the reference built for the host's full vector ISA
(x86-64-v4, AVX-512); the parity tests use the x86-64-v3 build.  Without
-ffast-math and with -ffp-contract=off, vectorisation may not change a
double: both builds must step to the same state bit for bit."""
import numpy as np
import pytest

from oracle import ref as R
from tests import helpers as H


def _avx512():
    try:
        with open("/proc/cpuinfo") as f:
            return "avx512f" in f.read()
    except OSError:
        return False


@pytest.mark.skipif(not _avx512(), reason="the host has no AVX-512")
@pytest.mark.parametrize("mhd", [True, False])
def test_timing_build_gives_the_parity_builds_doubles(mhd):
    states = []
    for variant in ("", "v4"):
        r = R.Reference(mhd, variant)
        p = R.params_fourier(root=2, nmodes=8, kmax=2) if mhd else R.params_sod(nblocks_x=8)
        r.setup(p)
        st = r.run(3)
        states.append((st, H.ref_state(r)))
    (st_a, (Wa, Ba)), (st_b, (Wb, Bb)) = states
    assert st_a == st_b
    assert H.same_values(Wa, Wb)
    if mhd:
        assert np.array_equal(Ba, Bb)
