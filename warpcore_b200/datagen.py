"""Seeded synthetic inputs generated on the device (the reference's
random_distributions.cuh:50-326 covers the same ground with kiss_rng, which
is not available here).

- unique_keys32 / unique_keys64: n distinct keys, none equal to the empty
  (0) or tombstone (all ones) sentinel.  They come from MurmurHash3's fmix,
  a bijection of the 32/64-bit index, so no sort or dedup is needed.
- uniform_values: independent uniform 32/64-bit values.
- zipf_ranks: Zipf(s) ranks by the rejection sampler that
  random_distributions.cuh:285-310 uses (a published method).  Ranks are
  0-based, so no index runs past the input.

Tensors are int32/int64 holding the unsigned bit patterns.
"""
import torch

MASK64 = (1 << 64) - 1


def _srl(x, s):
    return torch.bitwise_and(torch.bitwise_right_shift(x, s), (1 << (64 - s)) - 1)


def fmix64(x):
    """MurmurHash3 fmix64 on int64 tensors (two's complement wrap)"""
    c1 = 0xFF51AFD7ED558CCD - (1 << 64)
    c2 = 0xC4CEB9FE1A85EC53 - (1 << 64)
    x = torch.bitwise_xor(x, _srl(x, 33))
    x = x * c1
    x = torch.bitwise_xor(x, _srl(x, 33))
    x = x * c2
    x = torch.bitwise_xor(x, _srl(x, 33))
    return x


def _signed64(v):
    v &= MASK64
    return v - (1 << 64) if v >= (1 << 63) else v


def unique_keys64(start, n, seed, device="cuda"):
    off = _signed64(seed * 0x9E3779B97F4A7C15)
    idx = torch.arange(start, start + n + 4, dtype=torch.int64, device=device) + off
    k = fmix64(idx)
    k = k[(k != 0) & (k != -1)]
    return k[:n].contiguous()


def unique_keys32(start, n, seed, device="cuda"):
    idx = torch.arange(start, start + n + 4, dtype=torch.int64, device=device)
    x = (idx + seed * 0x9E3779B9) & 0xFFFFFFFF
    x = x ^ (x >> 16)
    x = (x * 0x85EBCA6B) & 0xFFFFFFFF
    x = x ^ (x >> 13)
    x = (x * 0xC2B2AE35) & 0xFFFFFFFF
    x = x ^ (x >> 16)
    x = x[(x != 0) & (x != 0xFFFFFFFF)][:n]
    return (x - ((x >= (1 << 31)).to(torch.int64) << 32)).to(torch.int32).contiguous()


def unique_keys(key_bytes, start, n, seed, device="cuda"):
    return (unique_keys32 if key_bytes == 4 else unique_keys64)(start, n, seed, device)


def uniform_values(n, nbytes, gen, device="cuda"):
    if nbytes == 8:
        return torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64,
                             device=device, generator=gen)
    return torch.randint(-(1 << 31), (1 << 31) - 1, (n,), dtype=torch.int32,
                         device=device, generator=gen)


def zipf_ranks(n_in, s, n_out, gen, device="cuda"):
    """Zipf(s) ranks in [0, n_in) by rejection sampling"""
    t = (float(n_in) ** (1.0 - s) - s) / (1.0 - s)
    out = torch.empty(n_out, dtype=torch.int64, device=device)
    filled = 0
    while filled < n_out:
        m = int((n_out - filled) * 1.3) + 1024
        p = torch.rand(m, dtype=torch.float64, device=device, generator=gen)
        y = torch.rand(m, dtype=torch.float64, device=device, generator=gen)
        pt = p * t
        inv_b = torch.where(pt <= 1.0, pt, torch.pow(pt * (1.0 - s) + s, 1.0 / (1.0 - s)))
        k = torch.floor(inv_b + 1.0)
        b = torch.where(k <= 1.0, torch.full_like(inv_b, 1.0 / t), torch.pow(inv_b, -s) / t)
        rat = torch.pow(k, -s) / (b * t)
        acc = k[y < rat].clamp(max=n_in).to(torch.int64) - 1
        take = min(acc.numel(), n_out - filled)
        out[filled:filled + take] = acc[:take]
        filled += take
    return out
