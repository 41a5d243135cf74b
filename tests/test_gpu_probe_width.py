"""Warp-cooperative lookups and deletes (CF_OPT_PROBE_WIDTH).

The reference's containsMany / deleteMany (CuckooFilter.cuh:1143-1183) probe a
key's buckets one thread per key.  With a probe width W > 1, W consecutive
lanes share a key, each loading its 4- or 8-byte piece of the bucket; a lookup
votes by ballot and a delete assembles the bucket's slot mask by shuffles and
clears the reference's slot with one compare-and-swap on the piece holding it.
Every supported width must give the one-lane results exactly:
  * lookups on a table image loaded from the oracle equal the oracle's;
  * deletes one key per call leave the oracle's image (the reference's slot);
  * a bulk delete removes every stored key it is given and leaves the same
    contents (each bucket's sorted tags) as the one-lane kernel;
  * widths a geometry cannot split into 4- or 8-byte lanes are refused.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import dev, host_u8, image, make  # noqa: E402


def widths(bits: int, bs: int) -> list[int]:
    bb = bits * bs // 8
    return [w for w in (2, 4, 8, 16, 32) if bb % w == 0 and bb // w in (4, 8) and bs <= 64]


CASES = [(8, 16, 16), (8, 8, 16), (8, 32, 8), (4, 16, 16), (8, 16, 4), (8, 8, 64), (8, 16, 32), (4, 32, 16),
         (8, 16, 64)]


def test_every_case_has_a_width():
    for _, bits, bs in CASES:
        assert widths(bits, bs), (bits, bs)


@pytest.mark.parametrize("kb,bits,bs", CASES)
def test_lookups_equal_the_oracle_at_every_width(cfb, orc, kb, bits, bs):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 16)
    try:
        pos = orc.splitmix64(61, int(0.93 * f.capacity()))
        neg = orc.splitmix64(62, 100_000)
        if kb == 4:
            pos, neg = pos.astype(np.uint32), neg.astype(np.uint32)
        o.insert(pos)
        f.load_table(torch.from_numpy(o.table).cuda())
        q = np.concatenate([pos, neg, pos[:7]])  # a length that is not a multiple of the keys per group
        want = o.contains(q, threads=4)
        for w in [1] + widths(bits, bs):
            f.setOption(cfb.OPT_PROBE_WIDTH, w)
            assert f.getOption(cfb.OPT_PROBE_WIDTH) == w
            got = host_u8(f.containsMany(dev(q)))
            assert np.array_equal(got, want), w
    finally:
        f.close()


@pytest.mark.parametrize("kb,bits,bs", [(8, 16, 16), (8, 8, 16), (8, 32, 8), (4, 16, 16), (8, 16, 64)])
def test_sequential_delete_bit_exact_at_every_width(cfb, orc, kb, bits, bs):
    for w in widths(bits, bs):
        f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 12)
        try:
            f.setOption(cfb.OPT_PROBE_WIDTH, w)
            keys = orc.splitmix64(65, int(0.9 * f.capacity()))
            if kb == 4:
                keys = keys.astype(np.uint32)
            o.insert(keys)
            f.load_table(torch.from_numpy(o.table).cuda())
            dels = np.concatenate([keys[::3], orc.splitmix64(66, 200).astype(keys.dtype), keys[:50]])
            d = dev(dels)
            out = torch.empty(1, dtype=torch.bool, device="cuda")
            got = np.empty(len(dels), np.uint8)
            for i in range(len(dels)):
                f.deleteMany(d[i:i + 1], out)
                got[i] = int(out.item())
            _, want = o.delete(dels)
            assert np.array_equal(got, want), w
            assert np.array_equal(image(f), o.table), w
            assert f.occupiedSlots() == o.occupied()
        finally:
            f.close()


def bucket_contents(img: np.ndarray, bits: int, bs: int) -> np.ndarray:
    slots = img.view({8: np.uint8, 16: np.uint16, 32: np.uint32}[bits]).reshape(-1, bs)
    return np.sort(slots, axis=1)


@pytest.mark.parametrize("kb,bits,bs", [(8, 16, 16), (8, 8, 16), (8, 32, 8), (4, 16, 16), (8, 8, 64)])
def test_bulk_delete_matches_one_lane(cfb, orc, kb, bits, bs):
    """Two batches on the same image at every width: half of the stored keys
    (each removes its own copy, so every per-key result is 1 and the contents
    left are the same for every width), then keys deleted already and keys
    never inserted that the oracle finds in neither bucket (every result 0,
    nothing removed: the not-found path of both buckets)."""
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 20)
    try:
        keys = orc.splitmix64(71, int(0.95 * f.capacity()))
        if kb == 4:
            keys = np.unique(keys.astype(np.uint32))
        o.insert(keys)
        src = torch.from_numpy(o.table).cuda()
        half = keys[: len(keys) // 2]
        o.delete(half)
        cand = np.concatenate([keys[:1000], orc.splitmix64(72, 50_000).astype(keys.dtype)])
        absent = cand[~o.contains(cand, threads=4).astype(bool)]
        assert len(absent) > 1000
        first, second = dev(half), dev(absent)
        contents = {}
        for w in [1] + widths(bits, bs):
            f.load_table(src)
            f.setOption(cfb.OPT_PROBE_WIDTH, w)
            out1 = torch.empty(first.numel(), dtype=torch.bool, device="cuda")
            occ1 = f.deleteMany(first, out1)
            assert host_u8(out1).all(), f"width {w}: a stored key could not be deleted"
            assert occ1 == f.countOccupiedSlots() == o.occupied()
            out2 = torch.ones(second.numel(), dtype=torch.bool, device="cuda")
            assert f.deleteMany(second, out2) == occ1
            assert not host_u8(out2).any(), w
            contents[w] = bucket_contents(image(f), bits, bs)
        for w, c in contents.items():
            assert np.array_equal(c, contents[1]), w
    finally:
        f.close()


def test_unsupported_widths_are_refused(cfb, orc):
    f, _ = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 12)
    g, _ = make(cfb, orc, 8, 16, 128, 0, 500, 1 << 14)
    try:
        for w in (2, 3, 6, 16, 64):  # 32-byte buckets: lanes of 16, 10.7, 5.3, 2 bytes; more than a warp
            with pytest.raises(cfb.CuckooError):
                f.setOption(cfb.OPT_PROBE_WIDTH, w)
            assert f.getOption(cfb.OPT_PROBE_WIDTH) == 0
        with pytest.raises(cfb.CuckooError):  # 128 slots: slot masks hold at most 64
            g.setOption(cfb.OPT_PROBE_WIDTH, 32)
    finally:
        f.close()
        g.close()
