"""gsb_dp_extend_static (the allocation-free variant of gsb_dp_extend) through the C ABI.

Collected last on purpose: it must pass both in a fresh process and after every other test has used the device.
Two calls in a row with different shapes check that the shared static scratch carries nothing from one call into
the next; both must equal gsb_dp_extend on the same inputs.
"""
import numpy as np
import pytest

TOL = 1e-12   # the same kernel on the same inputs: expected bit-identical


def _case(rng, r, rn, nker):
    positions = sorted(rng.choice(r + 1, size=rn, replace=False).tolist())
    ker = [int(rng.integers(1, 1 << (r + 1))) for _ in range(nker)]
    rho = int(rng.integers(0, 1 << r))
    wv = (complex(*rng.normal(size=2)), complex(*rng.normal(size=2)))
    old = rng.normal(size=1 << r) + 1j * rng.normal(size=1 << r)
    return old, positions, ker, rho, wv


@pytest.mark.gpu
def test_extend_static_equals_extend_on_two_calls():
    import gsb
    rng = np.random.default_rng(2024)
    for (r, rn, nker) in [(16, 16, 1), (11, 9, 2)]:
        old, piv, ker, rho, wv = _case(rng, r, rn, nker)
        want = gsb.dp_extend(old, r, rn, rho, piv, ker, wv)
        got = gsb.dp_extend_static(old, r, rn, rho, piv, ker, wv)
        assert got.shape == want.shape == (1 << rn,)
        assert np.max(np.abs(got - want)) <= TOL * max(1.0, np.max(np.abs(want)))


@pytest.mark.gpu
def test_extend_static_allocates_no_device_memory():
    """After the first call on the device (which looks up the scratch's address), further calls leave the device's
    free memory exactly as it was: they allocate nothing."""
    import torch
    import gsb
    rng = np.random.default_rng(11)
    old, piv, ker, rho, wv = _case(rng, 14, 14, 1)
    gsb.dp_extend_static(old, 14, 14, rho, piv, ker, wv)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        gsb.dp_extend_static(old, 14, 14, rho, piv, ker, wv)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


@pytest.mark.gpu
def test_extend_static_rejects_tables_beyond_its_scratch():
    import gsb
    rng = np.random.default_rng(5)
    old, piv, ker, rho, wv = _case(rng, 17, 16, 1)
    with pytest.raises(gsb.GsbError) as e:
        gsb.dp_extend_static(old, 17, 16, rho, piv, ker, wv)
    assert e.value.code == 1 and "static scratch" in str(e.value)
