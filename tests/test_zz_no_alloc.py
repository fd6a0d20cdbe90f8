"""ss_measure_corr_noalloc: the echo correlator over caller-owned device
vectors with its scratch in static device memory, checked against
ss_measure_corr (the engine entry point) on the same vectors.  Collected last
so that it also runs after every other test has used the device."""
import numpy as np
import pytest

import spin_systems_b200 as ss


def test_rejects_sizes_beyond_the_scratch():
    ss.load()
    for nspins in (0, 31, 64):
        with pytest.raises(ss.OutOfRangeError, match="nspins must be in"):
            ss.measure_corr_noalloc(0, 0, nspins, 0)


def _states(engine, nspins, seed):
    import torch
    rng = np.random.default_rng(seed)
    host = [rng.standard_normal(2 << nspins) for _ in range(2)]
    host = [h / np.linalg.norm(h) for h in host]
    psi, ref = (ss.StateVector(engine, nspins, h) for h in host)
    dev = [torch.from_numpy(h).to("cuda:0") for h in host]
    torch.cuda.synchronize()
    return psi, ref, dev


@pytest.mark.gpu
@pytest.mark.parametrize("nspins", [1, 5, 12, 21])
def test_matches_engine_correlator_twice_in_a_row(engine, nspins):
    psi, ref, (dpsi, dref) = _states(engine, nspins, 1000 + nspins)
    for axis in (0, 1, 2):
        want = ss.measure_corr(psi, ref, axis)
        got1 = ss.measure_corr_noalloc(dpsi.data_ptr(), dref.data_ptr(), nspins, axis)
        got2 = ss.measure_corr_noalloc(dpsi.data_ptr(), dref.data_ptr(), nspins, axis)
        assert got1 == want and got2 == want, (axis, got1, got2, want)


@pytest.mark.gpu
def test_caller_stream_and_no_device_allocation(engine):
    import torch
    nspins = 18
    psi, ref, (dpsi, dref) = _states(engine, nspins, 7)
    want = ss.measure_corr(psi, ref, 0)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    ss.measure_corr_noalloc(dpsi.data_ptr(), dref.data_ptr(), nspins, 0, side.cuda_stream)
    side.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    for _ in range(20):
        got = ss.measure_corr_noalloc(dpsi.data_ptr(), dref.data_ptr(), nspins, 0,
                                      side.cuda_stream)
        assert got == want
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0


@pytest.mark.gpu
def test_rejects_host_and_misaligned_pointers(engine):
    import torch
    host = np.zeros(2 << 4)
    dev = torch.zeros(2 << 4, dtype=torch.float64, device="cuda:0")
    with pytest.raises(ss.InvalidArgumentError, match="not device memory"):
        ss.measure_corr_noalloc(host.ctypes.data, dev.data_ptr(), 4, 2)
    with pytest.raises(ss.InvalidArgumentError, match="16-byte aligned"):
        ss.measure_corr_noalloc(dev.data_ptr() + 8, dev.data_ptr(), 4, 2)
    with pytest.raises(ss.InvalidArgumentError, match="null state"):
        ss.measure_corr_noalloc(0, dev.data_ptr(), 4, 2)


@pytest.mark.gpu
def test_rejects_a_vector_shorter_than_its_spin_count(engine):
    # One exact-size cudaMalloc of 64 KiB (torch's allocator would carve a
    # tensor out of a larger segment, which the check rightly accepts): a
    # pointer 8 KiB before its end cannot hold the 16 KiB of a 10-spin vector.
    from cuda.bindings import runtime as rt
    err, base = rt.cudaMalloc(1 << 16)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        rc, = rt.cudaMemset(base, 0, 1 << 16)
        assert rc == rt.cudaError_t.cudaSuccess
        tail = int(base) + (1 << 16) - 8192
        ok = int(base) + (1 << 16) - 16384
        with pytest.raises(ss.InvalidArgumentError, match="shorter than"):
            ss.measure_corr_noalloc(tail, ok, 10, 0)
        with pytest.raises(ss.InvalidArgumentError, match="shorter than"):
            ss.measure_corr_noalloc(ok, tail, 10, 0)
        assert ss.measure_corr_noalloc(ok, ok, 10, 2) == (0.0, 0.0)
    finally:
        rt.cudaFree(base)
