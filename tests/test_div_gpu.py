"""The batched face kernel divides with fused multiply-adds (FxDivFma in
fornaxamr_b200/csrc/fx_physics.cuh: Markstein's method, the correctly
rounded quotient without the general path's branches) wherever the operands
and the quotient lie in [2^-400, 2^401), and with native division elsewhere.
Bit parity with the reference rests on that quotient being the correctly
rounded one, so the device self-test compares it with native division on
17 billion seeded random pairs inside the range (random signs and
significands, the delicate significands 1.11...1, 1 and 1 + ulp, zero
dividends of either sign) and on a quarter billion pairs over the whole
exponent range, where it must either agree or hand the pair back."""
import ctypes as C

import pytest

import fornaxamr_b200 as fx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("emax,log2n", [(190, 34), (1022, 28)])
def test_fma_division_is_the_correctly_rounded_quotient(emax, log2n):
    L = fx.library()
    mism, out = C.c_ulonglong(0), C.c_ulonglong(0)
    rc = L.fx_selftest_div(0, 1 << log2n, 0x5EED0000 + emax, emax, C.byref(mism), C.byref(out))
    assert rc == 0
    print(f"exponents in [-{emax}, {emax}]: {1 << log2n} pairs, {out.value} outside the method's range, "
          f"{mism.value} differing quotients")
    assert mism.value == 0
    if emax == 190:
        # both operands within 2^+-191: the quotient is always in range
        assert out.value == 0
