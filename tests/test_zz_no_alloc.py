"""The all-pairs entry point that allocates nothing
(n_body_sim_pro_cuda_allpairs_acceleration_noalloc), through the C ABI.

It exists for callers that cannot allocate device memory (during CUDA graph
capture, inside frameworks that own every allocation, in loops that must not
touch the allocator); it keeps its working memory in a static device array
limited to 16384 particles.  Its output must agree with the allocating entry
point n_body_sim_pro_gravity_compute_acceleration_cuda and with the FP64
oracle (the reference's scalar all-pairs sum, gravity.c:15-70) within the
all-pairs tolerances of tests/test_allpairs_gpu.py, on calls in a row: the
first at exactly the 16384-particle limit, which fills the whole scratch
array, then smaller ones, so stale contents left in the shared array by an
earlier call must not leak into a later one.  This test allocates its own
device buffers with torch: it plays the caller, who owns inputs and outputs.

The file name sorts last so a stop-at-first-failure run has run every other
test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

RMS_TOL = 2e-6  # tests/test_allpairs_gpu.py
MAX_TOL = 5e-5  # against the allocating entry point: the same FP32 arithmetic
# against the FP64 oracle, the largest per-particle relative error comes from
# particles whose forces nearly cancel (tests/test_allpairs_gpu.py's precision
# study holds it to the same bound)
ORACLE_MAX_TOL = 5e-4


def _entry(nb):
    f = nb.library().n_body_sim_pro_cuda_allpairs_acceleration_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 7 + [C.c_size_t, C.c_double, C.c_double, C.c_void_p,
                                     C.POINTER(nb.Error)]
    return f


def _max_rel(a, ref):
    return float(np.max(np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)))


LIMIT = 16384  # particles: the static scratch array's capacity


def test_noalloc_matches_allocating_entry_point_and_oracle_on_calls_in_a_row(cuda):
    import torch

    noalloc = _entry(cuda)
    g = cuda.gravity_init(1.0, 0.01)
    side_stream = torch.cuda.Stream()
    for call, (n, seed) in enumerate(((LIMIT, 1), (9000, 2), (3000, 3))):
        p = O.preset("globular_cluster", n, seed)
        s = cuda.ParticleSystem(*[getattr(p, f).copy() for f in O.FIELDS])
        expected = cuda.n_body_sim_pro_gravity_compute_acceleration_cuda(s, g)
        oracle = O.gravity_reference(p.copy(), 1.0, 0.01, openmp=True)

        inputs = [torch.tensor(getattr(p, f), dtype=torch.float64, device="cuda")
                  for f in ("x", "y", "z", "m")]
        outputs = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
                   for _ in range(3)]
        torch.cuda.synchronize()
        stream = None if call == 0 else C.c_void_p(side_stream.cuda_stream)
        err = cuda.Error()
        rc = noalloc(*[t.data_ptr() for t in inputs + outputs], n, 1.0, 0.01, stream,
                     C.byref(err))
        assert rc == cuda.Status.OK, err.message
        torch.cuda.synchronize()
        got = np.stack([t.cpu().numpy() for t in outputs], axis=1)
        assert np.all(np.isfinite(got))
        assert O.rms_relative_error(got, expected) < RMS_TOL
        assert _max_rel(got, expected) < MAX_TOL
        assert O.rms_relative_error(got, oracle) < RMS_TOL
        assert _max_rel(got, oracle) < ORACLE_MAX_TOL


def test_noalloc_rejects_what_it_cannot_do(cuda):
    import torch

    noalloc = _entry(cuda)
    buf = torch.zeros(16385, dtype=torch.float64, device="cuda")
    ptrs = [buf.data_ptr()] * 7
    err = cuda.Error()
    assert noalloc(*ptrs, 16385, 1.0, 0.01, None, C.byref(err)) == cuda.Status.INVALID_ARGUMENT
    assert b"16384" in err.message
    host = np.zeros(16, dtype=np.float64)
    hptrs = [host.ctypes.data] * 7
    assert noalloc(*hptrs, 16, 1.0, 0.01, None, C.byref(err)) == cuda.Status.INVALID_ARGUMENT
    assert noalloc(*ptrs, 0, 1.0, 0.01, None, C.byref(err)) == cuda.Status.OK
