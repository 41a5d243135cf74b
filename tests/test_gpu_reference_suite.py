"""The reference's unit tests (tests/test_cuckoo_filter.cu, 12 gtest cases), run
against this library through its Python mirror of the reference API.

Configuration as in the reference fixture: CuckooConfig<uint32_t, 16, 500, 256,
16> (XOR policy, DFS eviction, uint64 words).  The reference draws keys from
std::mt19937(42) in [1, 2^32-1]; a seeded numpy generator over the same range
stands in for it.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TARGET_LOAD_FACTOR = 0.95


@pytest.fixture
def Config(cfb):
    return cfb.CuckooConfig(T="uint32_t", bitsPerTag=16, maxEvictions=500, blockSize=256, bucketSize=16)


@pytest.fixture
def rng():
    return np.random.Generator(np.random.MT19937(42))


def keys_dev(values):
    return torch.tensor(np.asarray(values, dtype=np.uint32).view(np.int32), device="cuda")


def random_keys(rng, n):
    return rng.integers(1, 2**32 - 1, size=n, dtype=np.uint64, endpoint=True).astype(np.uint32)


def out_u8(n):
    return torch.zeros(n, dtype=torch.uint8, device="cuda")


def host(t):
    return t.cpu().numpy()


def test_BasicInsertAndQuery(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    keys = [1, 2, 3, 4, 5, 100, 200, 300]
    d = keys_dev(keys)
    assert f.insertMany(d) == len(keys), "All keys should be inserted successfully"
    out = out_u8(len(keys))
    f.containsMany(d, out)
    assert host(out).all()


def test_EmptyFilter(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev([1, 2, 3, 4, 5])
    out = out_u8(5)
    f.containsMany(d, out)
    assert host(out).sum() == 0, "Empty filter should not find any keys"


def test_ClearOperation(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev([1, 2, 3, 4, 5])
    out = out_u8(5)
    f.insertMany(d)
    f.containsMany(d, out)
    assert host(out).all(), "Key should be found before clear"
    f.clear()
    f.containsMany(d, out)
    assert host(out).sum() == 0, "After clear, no keys should be found"
    assert f.loadFactor() == 0.0


def test_LoadFactor(cfb, Config, rng):
    f = cfb.CuckooFilter(Config, 10000)
    assert f.loadFactor() == 0.0
    d = keys_dev(random_keys(rng, 5000))
    inserted = f.insertMany(d)
    lf = f.loadFactor()
    assert 0.0 < lf <= 1.0
    assert lf == pytest.approx(np.float32(inserted) / np.float32(f.capacity()), rel=1e-6)
    assert inserted > 0


def test_NearCapacityInsertion(cfb, Config, rng):
    num_keys = int((1 << 20) * TARGET_LOAD_FACTOR)
    f = cfb.CuckooFilter(Config, num_keys)
    d = keys_dev(random_keys(rng, num_keys))
    out = out_u8(num_keys)
    inserted = f.insertMany(d)
    assert inserted > num_keys * 0.99, "Should insert at least 99% of keys"
    f.containsMany(d, out)
    assert host(out).sum() > inserted * 0.99, "Should find at least 99% of inserted keys"


def test_DuplicateInsertions(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev([1, 1, 2, 2, 3, 3, 4, 4, 5, 5])
    assert f.insertMany(d) == 10
    u = keys_dev([1, 2, 3, 4, 5])
    out = out_u8(5)
    f.containsMany(u, out)
    assert host(out).all()


def test_BasicDeletion(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    keys = [1, 2, 3, 4, 5, 100, 200, 300]
    d = keys_dev(keys)
    assert f.insertMany(d) == len(keys)
    out = out_u8(len(keys))
    f.containsMany(d, out)
    assert host(out).all()
    dout = out_u8(len(keys))
    remaining = f.deleteMany(d, dout)
    assert host(dout).all(), "every key should be deleted"
    assert remaining == 0, "No keys should remain after deletion"
    f.containsMany(d, out)
    assert host(out).sum() == 0


def test_DeleteNonExistentKeys(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev([1, 2, 3, 4, 5])
    dout = out_u8(5)
    f.deleteMany(d, dout)
    assert host(dout).sum() == 0


def test_PartialDeletion(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    assert f.insertMany(keys_dev(list(range(1, 11)))) == 10
    dk = keys_dev([2, 4, 6, 8, 10])
    dout = out_u8(5)
    remaining = f.deleteMany(dk, dout)
    assert host(dout).all()
    assert remaining == 5
    out = out_u8(5)
    f.containsMany(dk, out)
    assert host(out).sum() == 0
    f.containsMany(keys_dev([1, 3, 5, 7, 9]), out)
    assert host(out).all()


def test_DeleteAndReinsert(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev([1, 2, 3, 4, 5])
    out = out_u8(5)
    f.insertMany(d)
    f.deleteMany(d)
    f.containsMany(d, out)
    assert host(out).sum() == 0
    assert f.insertMany(d) == 5, "Should be able to reinsert deleted keys"
    f.containsMany(d, out)
    assert host(out).all()


def test_LoadFactorAfterDeletion(cfb, Config, rng):
    f = cfb.CuckooFilter(Config, 10000)
    d = keys_dev(random_keys(rng, 1000))
    f.insertMany(d)
    before = f.loadFactor()
    assert before > 0.0
    remaining = f.deleteMany(d)
    after = f.loadFactor()
    assert after < before
    assert after == pytest.approx(np.float32(remaining) / np.float32(f.capacity()), rel=1e-6)


def test_DeleteDuplicates(cfb, Config):
    f = cfb.CuckooFilter(Config, 10000)
    f.insertMany(keys_dev([1, 1, 1, 2, 2, 3]))
    dout = out_u8(3)
    f.deleteMany(keys_dev([1, 1, 1]), dout)
    assert host(dout).sum() >= 1
