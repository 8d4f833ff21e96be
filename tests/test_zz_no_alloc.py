"""kmm_xyzfft_noalloc (the physical -> spectral transform without device allocation) against the
context entry point kmm_xyzfft, through the C ABI.

The file name sorts last so that the check also runs after every other GPU test in the same
process (the library's file-scope scratch array is then shared with everything that ran before);
it passes alone in a fresh process as well.  Tolerance: the same kernels and twiddles run on both
paths, so the results agree to the routine tolerance of the parity tests (1e-12 relative).
"""

import numpy as np
import pytest

from polymer_dns_b200 import abi
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _context_transform(rt, p, phys):
    """kmm_xyzfft through a context: INITU -> U (reference layout, Fortran order)."""
    with rt.KmmContext(p) as g:
        g.upload("INITU", phys)
        g.call("xyzfft", "U", "INITU")
        return g.download("U")


def _noalloc_transform(rt, torch, p, phys, spec_dev):
    """kmm_xyzfft_noalloc on caller-owned device buffers; returns the spectral field."""
    src = torch.from_numpy(np.asfortranarray(phys).ravel(order="F")).cuda()
    spec_dev.fill_(float("nan"))   # every element must be written by the call
    stream = torch.cuda.current_stream()
    st = rt.xyzfft_noalloc(src.data_ptr(), spec_dev.data_ptr(), p.nx, p.ny, p.nz, stream.cuda_stream)
    assert st == abi.OK, abi.STATUS_NAMES.get(st, st)
    stream.synchronize()
    nyp, nxh = p.ny + 1, p.nx // 2
    out = spec_dev.cpu().numpy().view(np.complex128)
    return out.reshape((nyp, p.nz, nxh), order="F")


@pytest.mark.parametrize("grid", [(32, 32, 32), (24, 24, 16), (48, 40, 20)])
def test_noalloc_matches_context_transform(rt, grid):
    torch = pytest.importorskip("torch")
    p = kc.cfg_small(*grid)
    iu, iv, _ = kc.initial_fields(p)
    want_u = _context_transform(rt, p, iu)
    want_v = _context_transform(rt, p, iv)
    nspec = (p.ny + 1) * p.nz * (p.nx // 2)
    spec = torch.empty(2 * nspec, dtype=torch.float64, device="cuda")
    # two calls in a row on the same buffers, then a different field through the same scratch
    for _ in range(2):
        got = _noalloc_transform(rt, torch, p, iu, spec)
        assert np.all(np.isfinite(got))
        e = kc.rel_err(got, want_u)
        assert e <= TOL, "U rel err %.3e" % e
    e = kc.rel_err(_noalloc_transform(rt, torch, p, iv, spec), want_v)
    assert e <= TOL, "V rel err %.3e" % e


def test_noalloc_alternating_sizes(rt):
    """Changing the transform lengths between calls re-sends the twiddles; results stay exact."""
    torch = pytest.importorskip("torch")
    cases = []
    for grid in [(32, 32, 32), (24, 24, 16)]:
        p = kc.cfg_small(*grid)
        iu, _, _ = kc.initial_fields(p)
        spec = torch.empty(2 * (p.ny + 1) * p.nz * (p.nx // 2), dtype=torch.float64, device="cuda")
        cases.append((p, iu, _context_transform(rt, p, iu), spec))
    for _ in range(2):
        for p, iu, want, spec in cases:
            e = kc.rel_err(_noalloc_transform(rt, torch, p, iu, spec), want)
            assert e <= TOL, "grid %s rel err %.3e" % ((p.nx, p.ny, p.nz), e)


def test_noalloc_rejects_oversize_and_bad_lengths(rt):
    """Sizes beyond the fixed scratch, or lengths without an FFT plan, fail with KMM_ERR_ARG
    before any device work (the buffers passed are never touched)."""
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = buf.data_ptr()
    big = (256, 256, 128)   # (ny+1) nz nx = 8.4 M doubles > KMM_XYZFFT_NOALLOC_MAX
    assert (big[1] + 1) * big[2] * big[0] > 4 * 1024 * 1024
    assert rt.xyzfft_noalloc(ptr, ptr, *big) == abi.ERR_ARG
    assert rt.xyzfft_noalloc(ptr, ptr, 14, 16, 16) == abi.ERR_ARG    # nx = 14 has a factor 7
    assert rt.xyzfft_noalloc(ptr, ptr, 16, 16, 8192) == abi.ERR_ARG  # nz beyond the 4096 twiddles
    assert rt.xyzfft_noalloc(0, ptr, 16, 16, 16) == abi.ERR_ARG
    torch.cuda.synchronize()
    assert torch.count_nonzero(buf).item() == 0


def test_noalloc_allocates_no_device_memory(rt):
    """The property the entry point exists for: once the library's kernels are loaded (warm-up
    calls), further calls -- including ones at new grid sizes, which re-send the twiddles -- leave
    the device's free memory and torch's pool unchanged.  Every caller buffer is allocated before
    the measurement."""
    torch = pytest.importorskip("torch")
    grids = [(32, 32, 32), (24, 24, 16), (48, 40, 20), (40, 48, 24)]
    bufs = []
    for grid in grids:
        p = kc.cfg_small(*grid)
        iu, _, _ = kc.initial_fields(p)
        src = torch.from_numpy(np.asfortranarray(iu).ravel(order="F")).cuda()
        spec = torch.empty(2 * (p.ny + 1) * p.nz * (p.nx // 2), dtype=torch.float64, device="cuda")
        bufs.append((p, src, spec))
    stream = torch.cuda.current_stream()

    def call(p, src, spec):
        st = rt.xyzfft_noalloc(src.data_ptr(), spec.data_ptr(), p.nx, p.ny, p.nz, stream.cuda_stream)
        assert st == abi.OK, abi.STATUS_NAMES.get(st, st)

    for p, src, spec in bufs[:2]:     # warm-up: loads the kernels, resolves the array addresses
        call(p, src, spec)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(2):
        for p, src, spec in bufs:      # new lengths on the last two grids
            call(p, src, spec)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, "device free memory changed by %d bytes" % (free0 - free1)
    assert torch.cuda.memory_reserved() == reserved0
    assert all(bool(torch.isfinite(spec).all()) for _, _, spec in bufs)
