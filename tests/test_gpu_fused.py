"""The fused H.psi kernel (MCPI_OPT_FUSED_HPSI) against the two-kernel form.

The fused kernel runs exactly the arithmetic of the two kernels on the same
values, only in another schedule, so its output must be bitwise the same for
every schedule lead -- and both are checked against the
oracle's restatement of the reference (hamiltonianMatrix.h) on row samples.
A consumer's wait that runs out (producers held back by a test switch) must
end the kernel with MCPI_ERR_TIMEOUT and leave the space usable."""
import numpy as np
import pytest
import torch

import mcpi_b200 as mc
from conftest import rel

pytestmark = pytest.mark.gpu


def _space(N, M, g, fused, lead=0):
    sp = mc.FockSpace(N, M)
    sp.set_option(mc.OPT_DIRECT_HPSI, 0)       # the pair kernels, two or fused
    sp.set_option(mc.OPT_FUSED_HPSI, int(fused))
    sp.set_option(mc.OPT_FUSED_LEAD, lead)
    sp.set_integrals(*mc.lieb_integrals(M, g))
    return sp


def _state(nc, seed):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    x = torch.randn(nc, dtype=torch.complex128, device="cuda", generator=gen)
    return x / torch.linalg.vector_norm(x)


@pytest.mark.parametrize("N,M", [(16, 10), (10, 10), (7, 5), (2, 3), (9, 2), (6, 16), (12, 7)])
def test_fused_bitwise_equal_to_two_kernels(N, M):
    ref_sp = _space(N, M, 1.7, False)
    x = _state(ref_sp.nc, 100 + N + M)
    ref = ref_sp.apply_h(x)
    ref_sp.close()
    for lead in (0, 48, 128):
        sp = _space(N, M, 1.7, True, lead)
        for _ in range(2):       # the second call reuses the counters the first reset
            got = sp.apply_h(x)
            torch.cuda.synchronize()
            assert torch.equal(got, ref), (N, M, lead)
        sp.close()


def test_fused_against_oracle_rows(orc):
    N, M, g = 12, 9, 3.0
    sp = _space(N, M, g, True, 16)
    x = _state(sp.nc, 7)
    got = sp.apply_h(x).cpu().numpy()
    Ho, Hint = orc.lieb(M, g)
    IF = orc.focks(N, M)
    C = x.cpu().numpy()
    for r0 in (0, sp.nc // 3, sp.nc - 4000):
        want = orc.apply_h(N, M, C, Ho, Hint, mode=0, IF=IF, row0=r0, row1=r0 + 4000)
        assert rel(got[r0:r0 + 4000], want[r0:r0 + 4000]) <= 1e-12


def test_fused_lanczos_bitwise():
    N, M, lm = 12, 10, 40
    C0 = _state(mc.nc_of(N, M), 3).cpu().numpy()
    out = []
    for fused in (False, True):
        sp = _space(N, M, 2.0, fused, 16)
        it, diag, off, _ = sp.lanczos(C0, lm)
        out.append((it, diag.copy(), off.copy()))
        sp.close()
    assert out[0][0] == out[1][0] == lm
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_fused_wait_timeout_is_reported():
    N, M = 10, 8
    sp = _space(N, M, 1.0, True, 0)
    x = _state(sp.nc, 5)
    ref_sp = _space(N, M, 1.0, False)
    ref = ref_sp.apply_h(x)
    ref_sp.close()
    sp.set_option(mc.OPT_WAIT_LIMIT_KCYCLES, 1000)     # 1e6 cycles
    sp.set_option(mc.OPT_TEST_STALL_GATHER, 1)          # producers never publish
    sp.apply_h(x)
    with pytest.raises(mc.MCPIError) as ei:
        sp.sync()
    assert ei.value.status == 7                          # MCPI_ERR_TIMEOUT
    sp.set_option(mc.OPT_TEST_STALL_GATHER, 0)
    sp.set_option(mc.OPT_WAIT_LIMIT_KCYCLES, 0)
    got = sp.apply_h(x)
    sp.sync()
    assert torch.equal(got, ref)
    sp.close()
