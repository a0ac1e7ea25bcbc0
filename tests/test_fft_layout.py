"""The shared-memory layout of the register-radix transforms (csrc/fft.cuh), modelled on the
CPU: ``row_slot`` is a bijection on every row length used, and every pass's loads and
stores and the epilogues' bit-reversed reads cost the minimum number of shared-memory
wavefronts (32 four-byte banks; a warp's access needs 2 wavefronts for 8-byte and 4 for
16-byte elements).  The model restates row_slot, the pass decomposition and the access
pattern of ``dif_pass``."""

from collections import defaultdict

import pytest


def row_slot(i: int, bank_bits: int) -> int:
    """csrc/fft.cuh row_slot: the low bank_bits bits XORed with every higher group."""
    fold, shift = 0, bank_bits
    while shift < 16:
        fold ^= i >> shift
        shift += bank_bits
    return i ^ (fold & ((1 << bank_bits) - 1))


def wavefronts(slots, elem_bytes: int) -> int:
    """Wavefronts one warp access takes: the most distinct words any bank must serve."""
    banks = defaultdict(set)
    for s in slots:
        for w in range(elem_bytes // 4):
            word = (s * elem_bytes) // 4 + w
            banks[word % 32].add(word)
    return max(len(v) for v in banks.values())


def passes(log_n: int, radix_bits: int):
    """dif_pass's spans: radix_bits bits per pass, then the remainder in one pass."""
    out, log_len = [], log_n
    while log_len >= radix_bits:
        out.append((log_len, radix_bits))
        log_len -= radix_bits
    if log_len:
        out.append((log_len, log_len))
    return out


# (element bytes, bank bits, radix bits, row lengths): FP32 complex rows of 2^10..2^14
# points in one CTA, FP64 complex rows of 2^10..2^13 (and the clusters' sub-rows)
LAYOUTS = [(8, 4, 4, range(10, 15)), (16, 3, 3, range(10, 14))]


@pytest.mark.parametrize("elem,bank_bits,radix_bits,sizes", LAYOUTS)
def test_row_slot_is_a_bijection(elem, bank_bits, radix_bits, sizes):
    for log_n in sizes:
        n = 1 << log_n
        assert sorted(row_slot(i, bank_bits) for i in range(n)) == list(range(n))


@pytest.mark.parametrize("elem,bank_bits,radix_bits,sizes", LAYOUTS)
def test_every_access_takes_the_minimum_wavefronts(elem, bank_bits, radix_bits, sizes):
    ideal = elem * 32 // 128
    for log_n in sizes:
        n = 1 << log_n
        for log_len, k in passes(log_n, radix_bits):
            q = 1 << (log_len - k)
            for r in range(1 << k):  # the r-th load (and store) of every thread
                for w0 in range(0, n >> k, 32):
                    slots = []
                    for p in range(w0, min(w0 + 32, n >> k)):
                        j = p & (q - 1)
                        base = ((p >> (log_len - k)) << log_len) + j
                        slots.append(row_slot(base + r * q, bank_bits))
                    assert wavefronts(slots, elem) == ideal, (log_n, log_len, r, w0)
        # the epilogues read X[k] at row_slot(bitrev(k)) for consecutive k across a warp
        def bitrev(x):
            return int(format(x, f"0{log_n}b")[::-1], 2)
        for w0 in range(0, n, 32):
            assert wavefronts([row_slot(bitrev(x), bank_bits) for x in range(w0, w0 + 32)], elem) == ideal


def test_padding_alone_would_conflict():
    """The layout it replaced: one element of padding per 128 bytes leaves the bit-reversed
    reads many-way conflicted (why the swizzle exists)."""
    log_n = 14
    def bitrev(x):
        return int(format(x, f"0{log_n}b")[::-1], 2)
    padded = [bitrev(x) + (bitrev(x) >> 4) for x in range(32)]
    assert wavefronts(padded, 8) > 2
