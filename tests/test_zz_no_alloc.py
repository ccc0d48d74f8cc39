"""The allocation-free entry point, bp_beamform_max_noalloc.

It exists for callers that may not allocate device memory while they run
(a service that sets aside its GPU memory at start-up, or a host program
whose allocator owns the device): its working memory is a fixed array
compiled into the library.  This file is named so that pytest collects it
last.  The test calls the entry point several times in a row through the
C-ABI, on different problems, and checks each result bit for bit against the
existing allocating entry point, bp_beamform_max_direct_dev, and against the
CPU oracle -- the later calls also show that the previous call's leftovers
in the shared array do not leak into the next result.  The last problem
leaves samples without any candidate source (strict rule): there the output
keeps the caller's fill value and the argmax is 0, as in the reference.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(seed, N, S, P, T, dmax, dmin=0):
    rng = np.random.default_rng(seed)
    U = np.abs(rng.standard_normal((S, T, P))).astype(np.float32)
    D = rng.integers(dmin, dmax + 1, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.25, 2.0, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < 0.2] = 0.0
    return U, D, W


def _no_candidate_tail():
    """Strict rule, every weighted delay >= 600: samples t >= T - 600 have
    no candidate source; a tenth of the sources have no weighted station."""
    U, D, W = _problem(3, 500, 6, 2, 2000, 900, dmin=600)
    W[::10] = 0.0
    return U, D, W


def _expected(orc, oracle_lib, U, D, W, oob, fill):
    """The oracle's max/argmax with the caller's fill kept where no source
    is a candidate (strict rule: no weighted station or a delay out of the
    record; flexible rule: every sample of a non-empty grid has one)."""
    bm, am = oracle_lib.beamform_max(U, D, W, oob)
    T = U.shape[1]
    if oob == 0:
        mm = orc.fp64_minmax(D, W)
        t = np.arange(T)[None, :]
        lo, hi = mm[:, 0][:, None], mm[:, 1][:, None]
        has = ((lo <= hi) & (t + lo >= 0) & (t + hi < T)).any(axis=0)
    else:
        has = np.full(T, D.shape[0] > 0)
    return np.where(has, bm, np.float32(fill)), np.where(has, am, 0), has


def _rows(torch, U, pitch):
    """(S, T, P) prestacked traces -> (S * P, pitch) rows, zero padded."""
    S, T, P = U.shape
    rows = torch.zeros((S * P, pitch), dtype=torch.float32, device="cuda")
    rows[:, :T] = torch.from_numpy(U).cuda().permute(0, 2, 1).reshape(S * P, T)
    return rows


def test_noalloc_matches_allocating_entry_point_twice(orc, oracle_lib):
    import torch
    import beampower_b200 as bp
    from beampower_b200.tables import _stream_ptr

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    lib = bp.load_library("gpu")
    # the larger problem first, then smaller ones over the same array
    cases = [(_problem(1, 3000, 7, 2, 20000, 400), 1),
             (_problem(2, 700, 5, 2, 3000, 900), 0),
             (_no_candidate_tail(), 0)]
    for (U, D, W), oob in cases:
        S, T, P = U.shape
        N = D.shape[0]
        pitch = ((T + 63) // 64) * 64
        rows = _rows(torch, U, pitch)
        d = torch.from_numpy(D).cuda()
        w = torch.from_numpy(W).cuda()
        st = _stream_ptr()

        bm_a = torch.full((T,), -1.0, dtype=torch.float32, device="cuda")
        am_a = torch.full((T,), -1, dtype=torch.int32, device="cuda")
        rc = lib.bp_beamform_max_noalloc(rows.data_ptr(), T, 0, pitch, d.data_ptr(),
                                         w.data_ptr(), N, S, P, oob, bm_a.data_ptr(),
                                         am_a.data_ptr(), st)
        assert rc == 0

        bm_b = torch.full((T,), -1.0, dtype=torch.float32, device="cuda")
        am_b = torch.full((T,), -1, dtype=torch.int32, device="cuda")
        keys = torch.empty(T, dtype=torch.int64, device="cuda")
        rc = lib.bp_beamform_max_direct_dev(rows.data_ptr(), 0, None, T, 0, pitch,
                                            d.data_ptr(), w.data_ptr(), N, S, P, oob,
                                            keys.data_ptr(), bm_b.data_ptr(), am_b.data_ptr(),
                                            st)
        assert rc == 0, lib.bp_last_error()
        torch.cuda.synchronize()
        # FP32 results of the two entry points agree bit for bit
        assert torch.equal(bm_a.view(torch.int32), bm_b.view(torch.int32))
        assert torch.equal(am_a, am_b)
        # and equal the oracle's, the fill kept where no source is a candidate
        want_bm, want_am, has = _expected(orc, oracle_lib, U, D, W, oob, -1.0)
        got_bm, got_am = bm_a.cpu().numpy(), am_a.cpu().numpy()
        assert np.array_equal(got_bm.view(np.uint32), want_bm.view(np.uint32))
        assert np.array_equal(got_am, want_am)
    assert not has.all() and has.any()  # the last case has samples without candidates


def test_noalloc_rejects_sizes_beyond_its_fixed_array():
    import beampower_b200 as bp
    lib = bp.load_library("gpu")
    too_long = 524288 + 1
    assert lib.bp_beamform_max_noalloc(None, too_long, 0, too_long, None, None, 10, 2, 2, 0,
                                       None, None, None) == 6
    assert b"scratch" in lib.bp_last_error()
    assert lib.bp_beamform_max_noalloc(None, 100, 0, 100, None, None, 524288 + 1, 2, 2, 0,
                                       None, None, None) == 6
    assert b"scratch" in lib.bp_last_error()
