"""On-device input generators (random_distributions.cuh:50-326) against the
oracle: uniform words and distinct keys bit for bit (including seeds that
put a sentinel's preimage inside the range, so the skip is exercised), and
Zipf draws stream for stream, up to the last-bit differences of the
device's and the host's pow() near the acceptance boundary; the Zipf
frequencies are also checked against the distribution."""
import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import host

pytestmark = pytest.mark.gpu

GOLDEN = 0x9E3779B97F4A7C15


def _fmix_inverse(key, bits):
    """preimage under MurmurHash3's fmix (test helper, independent of the
    library's host code)"""
    mask = (1 << bits) - 1

    def unxs(y, r):
        x = y
        for _ in range(bits // r + 1):
            x = y ^ (x >> r)
        return x & mask

    if bits == 32:
        x = unxs(key & mask, 16)
        x = (x * pow(0xC2B2AE35, -1, 1 << 32)) & mask
        x = unxs(x, 13)
        x = (x * pow(0x85EBCA6B, -1, 1 << 32)) & mask
        return unxs(x, 16)
    x = unxs(key, 33)
    x = (x * pow(0xC4CEB9FE1A85EC53, -1, 1 << 64)) & mask
    x = unxs(x, 33)
    x = (x * pow(0xFF51AFD7ED558CCD, -1, 1 << 64)) & mask
    return unxs(x, 33)


def _seed_for_skip(bits, sentinel, index):
    """a seed whose key sequence hits `sentinel` at position `index`"""
    mask = (1 << bits) - 1
    g = GOLDEN & mask
    return ((_fmix_inverse(sentinel, bits) - index) * pow(g, -1, 1 << bits)) & mask


def _dev(n, nbytes):
    return torch.empty(n, dtype=torch.int32 if nbytes == 4 else torch.int64, device="cuda")


@pytest.mark.parametrize("nbytes", [4, 8])
@pytest.mark.parametrize("n", [0, 1, 1000, 1 << 20])
def test_uniform_matches_oracle(nbytes, n):
    out = wc.gen_uniform(_dev(n, nbytes), 12345)
    assert np.array_equal(host(out), o.gen_uniform(nbytes, n, 12345))


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("seed_kind", ["plain", "skip_empty", "skip_tombstone"])
def test_unique_matches_oracle(kb, seed_kind):
    bits = 8 * kb
    seed = {"plain": 99,
            "skip_empty": _seed_for_skip(bits, 0, 5),
            "skip_tombstone": _seed_for_skip(bits, (1 << bits) - 1, 700)}[seed_kind]
    n = 5000
    got = host(wc.gen_unique(_dev(n, kb), seed))
    want = o.gen_unique_keys(kb, n, seed)
    assert np.array_equal(got, want)
    assert np.unique(got).size == n
    assert not np.any((got == 0) | (got == (1 << bits) - 1))


@pytest.mark.parametrize("kb", [4, 8])
def test_unique_large_is_distinct(kb):
    n = 1 << 24
    out = wc.gen_unique(_dev(n, kb), 7)
    assert torch.unique(out).numel() == n
    assert not bool(((out == 0) | (out == -1)).any())
    # the start of the sequence equals the oracle's
    assert np.array_equal(host(out[:4096]), o.gen_unique_keys(kb, 4096, 7))


@pytest.mark.parametrize("nbytes", [4, 8])
@pytest.mark.parametrize("s", [0.5, 1.1, 2.0])
def test_zipf_matches_oracle_streams(nbytes, s):
    n_in, n_out = 1 << 16, 1 << 16
    got = host(wc.gen_zipf(_dev(n_out, nbytes), n_in, s, 4321))
    want = o.gen_zipf_streams(n_in, s, n_out, 4321, key_bytes=nbytes)
    assert got.min() >= 1 and got.max() <= n_in
    # device and host pow() may differ in the last bit; a draw decided that
    # close to its acceptance bound is rare
    assert int((got != want).sum()) <= 2


def test_zipf_from_input_array_and_frequencies():
    n_in, n_out, s = 1000, 1 << 22, 1.1
    keys = wc.gen_unique(_dev(n_in, 8), 3)
    out = wc.gen_zipf(_dev(n_out, 8), n_in, s, 11, in_=keys)
    ranks = wc.gen_zipf(_dev(n_out, 8), n_in, s, 11)
    assert torch.equal(out, keys[ranks - 1])
    # rank frequencies follow k^-s / H(n_in, s) (chi-square over the head)
    cnt = torch.bincount(ranks, minlength=n_in + 1)[1:].double().cpu().numpy()
    k = np.arange(1, n_in + 1, dtype=np.float64)
    p = k ** -s / np.sum(k ** -s)
    exp = p * n_out
    head = exp > 50
    chi2 = float(np.sum((cnt[head] - exp[head]) ** 2 / exp[head]))
    dof = int(head.sum()) - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_generator_errors():
    with pytest.raises(wc.WarpcoreError):
        wc.gen_zipf(_dev(10, 8), 100, 1.0, 1)
    with pytest.raises(wc.WarpcoreError):
        wc.gen_zipf(_dev(10, 8), 0, 1.5, 1)
    with pytest.raises(wc.WarpcoreError):
        wc.gen_uniform(torch.empty(4, dtype=torch.int16, device="cuda"), 1)
