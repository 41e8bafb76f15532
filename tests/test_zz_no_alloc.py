"""fp_solve_csr_upper_noalloc: the allocation-free CSR solve.

The entry point keeps its work vectors in one fixed device array shared by
every call, so these tests run two different systems back to back (a large one
first, then a small one, so a stale vector from the first call would show in
the second) and compare each with fp_solve_csr_upper, which allocates its own
buffers.  This file is collected last and also passes on its own.
"""
import re

import numpy as np
import pytest

from conftest import ROOT, rel_l2


def test_noalloc_limit_matches_header():
    from fluidprjct_b200 import capi
    hdr = open(f"{ROOT}/include/fluidprjct.h").read()
    m = re.search(r"#define FP_NOALLOC_MAX_N \(1 << (\d+)\)", hdr)
    assert m and capi.FP_NOALLOC_MAX_N == 1 << int(m.group(1))


def _poisson(O, W, H, D, obstacle):
    from fluidprjct_b200.scenes import box_3d
    lab = box_3d(W, H, D, 0.1, 0.55, 0.45, 0.5)
    if obstacle:
        lab[D // 2, H // 4, W // 3] = 0
    off, cols, vals = O.build_csr_upper(lab)
    return np.asarray(off, np.int32), np.asarray(cols, np.int32), np.asarray(vals, np.float64)


def _device_solve(off, cols, vals, b, tol):
    import torch
    from fluidprjct_b200 import capi
    dev = torch.device("cuda:0")
    t_off = torch.from_numpy(off).to(dev)
    t_cols = torch.from_numpy(cols).to(dev)
    t_vals = torch.from_numpy(vals).to(dev)
    t_b = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    t_x = torch.full_like(t_b, float("nan"))  # the call must overwrite every entry
    stream = torch.cuda.current_stream(dev).cuda_stream
    it, rr = capi.solve_csr_upper_noalloc(len(b), t_off.data_ptr(), t_cols.data_ptr(), t_vals.data_ptr(),
                                          t_b.data_ptr(), t_x.data_ptr(), tol=tol, max_iters=20000, stream=stream)
    torch.cuda.synchronize(dev)
    return t_x.cpu().numpy(), it, rr


@pytest.mark.gpu
def test_noalloc_matches_allocating_solve_on_two_calls(O, golden):
    from fluidprjct_b200 import capi
    rng = np.random.default_rng(7)
    big = _poisson(O, 40, 36, 32, obstacle=True)
    small = _poisson(O, 9, 8, 7, obstacle=False)
    tol = 1e-12
    for off, cols, vals in (big, small):
        n = len(off) - 1
        assert 0 < n <= capi.FP_NOALLOC_MAX_N
        b = rng.standard_normal(n)
        x_na, it_na, rr_na = _device_solve(off, cols, vals, b, tol)
        x_ref, it_ref, rr_ref = capi.solve_csr_upper(off, cols, vals, b, tol=tol, max_iters=20000)
        assert np.isfinite(x_na).all()
        assert rr_na <= tol and rr_ref <= tol
        assert abs(it_na - it_ref) <= 2
        assert rel_l2(x_na, x_ref) <= 1e-9
    # the known-answer system of the reference's test.cu, twice in a row
    kat = golden["kat"]
    for _ in range(2):
        x, it, rr = _device_solve(np.asarray(kat["offsets"], np.int32), np.asarray(kat["cols"], np.int32),
                                  np.asarray(kat["vals"], np.float64), np.asarray(kat["b"]), 1e-15)
        assert np.max(np.abs(x - np.asarray(kat["x"]))) <= 1e-12


@pytest.mark.gpu
def test_noalloc_leaves_device_free_memory_unchanged(O):
    """The call allocates nothing: after a first call (which looks up the
    scratch array's address), the device's free memory is the same after
    each of three more calls as before them."""
    import torch
    off, cols, vals = _poisson(O, 30, 28, 26, obstacle=True)
    b = np.random.default_rng(3).standard_normal(len(off) - 1)
    _device_solve(off, cols, vals, b, 1e-10)
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (off, cols, vals, b)]
    t_x = torch.zeros_like(t[3])
    torch.cuda.synchronize(dev)
    from fluidprjct_b200 import capi
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        capi.solve_csr_upper_noalloc(len(b), t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(),
                                     t_x.data_ptr(), tol=1e-10, max_iters=20000,
                                     stream=torch.cuda.current_stream(dev).cuda_stream)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, (free0, free1)


@pytest.mark.gpu
def test_noalloc_rejects_oversize_and_malformed():
    import torch
    from fluidprjct_b200 import capi
    dev = torch.device("cuda:0")
    off = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    vals = torch.ones(2, dtype=torch.float64, device=dev)
    b = torch.ones(2, dtype=torch.float64, device=dev)
    x = torch.zeros(2, dtype=torch.float64, device=dev)
    cols_ok = torch.tensor([0, 1], dtype=torch.int32, device=dev)
    cols_bad = torch.tensor([0, 2], dtype=torch.int32, device=dev)
    ptrs = lambda cols: (off.data_ptr(), cols.data_ptr(), vals.data_ptr(), b.data_ptr(), x.data_ptr())
    # too large: rejected before any of the buffers is touched
    with pytest.raises(capi.FluidError) as e:
        capi.solve_csr_upper_noalloc(capi.FP_NOALLOC_MAX_N + 1, *ptrs(cols_ok))
    assert e.value.code == capi.FP_ERR_ARG
    # a column index outside [0, n): found by the device-side check, no solve runs
    with pytest.raises(capi.FluidError) as e:
        capi.solve_csr_upper_noalloc(2, *ptrs(cols_bad))
    assert e.value.code == capi.FP_ERR_ARG
    # the identity afterwards: the rejected calls left nothing behind
    it, rr = capi.solve_csr_upper_noalloc(2, *ptrs(cols_ok), tol=1e-14)
    torch.cuda.synchronize(dev)
    assert torch.equal(x.cpu(), torch.ones(2, dtype=torch.float64)) and it <= 1


@pytest.mark.gpu
def test_noalloc_calls_from_two_threads_take_turns(O):
    """Two host threads, each on its own stream, solve different systems three
    times each at once.  ctypes releases the GIL during the call, so the calls
    overlap on the host; the per-device lock serialises them on the shared
    scratch, and every answer matches the allocating solve."""
    import threading

    import torch
    from fluidprjct_b200 import capi
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(11)
    systems = [_poisson(O, 30, 28, 26, obstacle=True), _poisson(O, 24, 20, 18, obstacle=False)]
    jobs = []
    for off, cols, vals in systems:
        b = rng.standard_normal(len(off) - 1)
        x_ref, _, _ = capi.solve_csr_upper(off, cols, vals, b, tol=1e-12, max_iters=20000)
        t = [torch.from_numpy(a).to(dev) for a in (off, cols, vals, np.ascontiguousarray(b, np.float64))]
        jobs.append((t, x_ref))
    torch.cuda.synchronize(dev)
    results = [[] for _ in jobs]
    errors = []

    def work(j):
        try:
            (t_off, t_cols, t_vals, t_b), _ = jobs[j]
            s = torch.cuda.Stream(dev)
            for _ in range(3):
                t_x = torch.full_like(t_b, float("nan"))
                torch.cuda.synchronize(dev)
                it, rr = capi.solve_csr_upper_noalloc(len(t_b), t_off.data_ptr(), t_cols.data_ptr(),
                                                      t_vals.data_ptr(), t_b.data_ptr(), t_x.data_ptr(),
                                                      tol=1e-12, max_iters=20000, stream=s.cuda_stream)
                results[j].append((t_x.cpu().numpy(), rr))
        except Exception as e:  # reported by the main thread
            errors.append(e)

    threads = [threading.Thread(target=work, args=(j,)) for j in range(len(jobs))]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=120)
    assert not errors and not any(th.is_alive() for th in threads)
    for (_, x_ref), res in zip(jobs, results):
        assert len(res) == 3
        for x, rr in res:
            assert rr <= 1e-12 and rel_l2(x, x_ref) <= 1e-9
