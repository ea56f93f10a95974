"""Column passes staged by TMA (cp.async.bulk.tensor tile loads and stores):
every product equals GMP's and the same product with the tiles staged by
cp.async, over transform classes whose column tiles have 16 to 128 columns,
odd and power-of-two first passes, products and squares; the launches of the
batch are the TMA kernels, and no bounded wait gave up."""
import json

import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

JK_FWD_TMA, JK_REV_TMA = 8, 9


@pytest.fixture
def tuning(gpu_lib):
    old = gpu_lib.get_tuning()
    yield gpu_lib
    gpu_lib.set_tuning(old)


def _set(gpu_lib, **kw):
    t = json.loads(gpu_lib.get_tuning())
    t.update(kw)
    t["overrides"] = kw.get("overrides", [])
    gpu_lib.set_tuning(json.dumps(t))


def _run_batch(gpu_lib, pairs):
    """All pairs as one device batch (graph replay); returns (results, launch kind codes)."""
    items, outs, keep = [], [], []
    for a, b in pairs:
        da = torch.from_numpy(a).cuda()
        db = None if b is None else torch.from_numpy(b).cuda()
        n = a.size if b is None else b.size
        r = torch.zeros(a.size + n, dtype=torch.uint64, device="cuda")
        keep.append((da, db))
        outs.append(r)
        items.append((r, da, db, a.size, n, O.magnitude_bits(a), 0 if b is None else O.magnitude_bits(b)))
    descs = gpu_lib.make_descs(items)
    torch.cuda.synchronize()
    bt = gpu_lib.Batch(descs)
    kinds = [s["code"] for s in bt.stats()]
    bt.run(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    res = [r.cpu().numpy() for r in outs]
    bt.close()
    return res, kinds


def _shapes(rng):
    pairs = []
    for m, n in ((65536, 65536), (60000, 20000), (30000, 30000), (131072, 100000), (200000, 190000)):
        pairs.append((rand_limbs(rng, m), rand_limbs(rng, n)))
    for m in (65536, 100000, 250000):
        pairs.append((rand_limbs(rng, m), None))
    pairs.append((np.full(90000, 2**64 - 1, dtype=np.uint64), np.full(90000, 2**64 - 1, dtype=np.uint64)))
    pairs.append((adversarial(rng, 70000), adversarial(rng, 50000)))
    return pairs


@pytest.mark.parametrize("tile_target", [4096, 8192])
def test_tma_column_passes_match_gmp_and_cp_async(tuning, tile_target):
    rng = np.random.default_rng(900 + tile_target)
    pairs = _shapes(rng)
    _set(tuning, tile_target=tile_target, tma=1)
    got, kinds = _run_batch(tuning, pairs)
    assert JK_FWD_TMA in kinds and JK_REV_TMA in kinds
    _set(tuning, tile_target=tile_target, tma=0)
    ref, kinds0 = _run_batch(tuning, pairs)
    assert JK_FWD_TMA not in kinds0
    for (a, b), g, r in zip(pairs, got, ref):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(g, want)
        assert np.array_equal(r, want)
    assert tuning.device_faults() == 0


def test_tma_single_products_and_forced_splits(tuning):
    rng = np.random.default_rng(911)
    a, b = rand_limbs(rng, 2**20), rand_limbs(rng, 2**20 - 5000)
    want = O.gmp_mul(a, b)
    _set(tuning, tile_target=4096, tma=1)
    assert np.array_equal(tuning.mul(a, b), want)
    assert np.array_equal(tuning.sqr(a), O.gmp_sqr(a))
    # several column passes of one radix-16 round each, TMA staged
    bch, N = tuning.ntt_params(O.magnitude_bits(a), O.magnitude_bits(b))
    S = len(tuning.plan_layout(N)["stages"])
    ends = list(range(1, S - 4, 2)) + [S - 1]
    _set(tuning, tile_target=4096, tma=1, overrides=[{"N": N, "sqr": 0, "pass_ends": ends, "tile_target": 4096}])
    assert np.array_equal(tuning.mul(a, b), want)
    assert tuning.device_faults() == 0
