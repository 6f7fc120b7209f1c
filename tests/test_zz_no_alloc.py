"""GPU test of ll_step_static, the entry point for callers that cannot
allocate device memory (an arena or pool owns it all, a host application
forbids allocation inside work calls, a loop must stay off the allocator).

It runs on device buffers the caller provides; its scratch is one static
array inside the library.  This test calls it through the C ABI twice in a
row (the second call continues from the first call's output) and checks both
outputs against the context-based entry points (ll_load_digits + ll_step)
on the same input: digit vectors equal after canonicalisation (exact integer
parity, as in the other GPU tests), and the same max roundoff error.  The
file name makes pytest collect it last."""
import ctypes

import numpy as np
import pytest

import cudalucas_b200 as cl
from cudalucas_b200 import native

pytestmark = pytest.mark.gpu


def static_step(q, n, offset, iters, d_in, d_out):
    err = ctypes.c_float(-1.0)
    rc = native.lib().ll_step_static(0, q, n, offset, iters, ctypes.c_void_p(d_in.data_ptr()),
                                     ctypes.c_void_p(d_out.data_ptr()), ctypes.byref(err), None)
    return rc, err.value


@pytest.mark.parametrize("q,n,k1,k2", [(86243, 4096, 300, 700), (216091, 12288, 500, 250),
                                       (1257787, 65536, 120, 80),
                                       (18454939, 1 << 20, 30, 20)])  # the stated maximum size
def test_static_entry_point_matches_context_entry_point(q, n, k1, k2):
    import torch
    off0 = (q * 3) // 7
    # the static entry point runs the two-launch kernels: so does the reference
    # context (short lengths would otherwise take the cluster-resident path, whose
    # roundoff maximum differs in its last bits)
    with cl.LLContext(q, n, tuning={"kernels": native.LL_KERNELS_NO_CLUSTER}) as c:
        c.start(off0)
        d0, o0 = c.read_digits()
        e1 = c.step(k1, report=True)
        d1, o1 = c.read_digits()
        # The static entry point starts every call from loaded digits.  A
        # context that goes on after a report step starts from the report
        # pass's own floating-point state, which another kernel instantiation
        # computes and which can differ in the last bits (same digits, a
        # different roundoff maximum on the next iteration); so the reference
        # reloads its digits too.
        c.load_digits(d1, o1)
        e2 = c.step(k2, report=True)
        d2, o2 = c.read_digits()
    dev_in = torch.from_numpy(d0.copy()).cuda()
    dev_mid = torch.zeros(n, dtype=torch.int32, device="cuda")
    dev_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc, s1 = static_step(q, n, o0, k1, dev_in, dev_mid)
    assert rc == 0
    rc, s2 = static_step(q, n, o1, k2, dev_mid, dev_out)
    assert rc == 0
    m1 = dev_mid.cpu().numpy()
    m2 = dev_out.cpu().numpy()
    assert np.array_equal(cl.standardize(m1, q, n)[0], cl.standardize(d1, q, n)[0])
    assert np.array_equal(cl.standardize(m2, q, n)[0], cl.standardize(d2, q, n)[0])
    assert cl.digits_res64(m2, q, n, o2) == cl.digits_res64(d2, q, n, o2)
    assert abs(s1 - e1) <= 1e-6 and abs(s2 - e2) <= 1e-6, (s1, e1, s2, e2)


def test_static_entry_point_rejects_sizes_beyond_its_maximum():
    import torch
    n = 2 * native.LL_STATIC_MAX_WORDS
    q = 40000003
    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc, _ = static_step(q, n, 0, 1, d, d)
    assert rc == native.LL_ERR_ARG


@pytest.mark.parametrize("q,n", [(86243, 4096),      # generic kernels
                                 (216091, 12288),    # specialised wide pass, generic tall pass
                                 (1257787, 65536)])  # specialised passes
def test_static_entry_point_reports_words_beyond_fp64_range(q, n):
    """Digits far outside the balanced range make the squared words exceed
    2^51, where a double has no fraction bits left for the roundoff reading.
    The kernels flag it, and the call reports the largest possible error (as
    ll_step does) so that a caller's roundoff policy rejects the result."""
    import torch
    d = torch.full((n,), 1 << 29, dtype=torch.int32, device="cuda")
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    for k in (1, 2):
        rc, err = static_step(q, n, 5, k, d, out)
        assert rc == 0
        assert err == 1.0, (k, err)
    # a valid state afterwards is unaffected by the shared scratch's contents
    with cl.LLContext(q, n) as c:
        c.start(5)
        d0, o0 = c.read_digits()
        c.step(40, report=True)
        want = c.res64()
    rc, err = static_step(q, n, o0, 40, torch.from_numpy(d0.copy()).cuda(), out)
    assert rc == 0 and err < 0.4
    assert cl.digits_res64(out.cpu().numpy(), q, n, c_offset(q, o0, 40)) == want


def c_offset(q, off, k):
    for _ in range(k):
        off = (2 * off) % q
    return off
