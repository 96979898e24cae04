"""Radiance cache on the GPU against the numpy oracle (oracle/radiance_cache.py): the hash-grid
encoding bit for bit, the tensor-core MLP forward pass and its gradients within the stated
BF16 tolerances, Adam step for step, and training that lowers the loss."""
import numpy as np
import pytest

import radiance_cache as rc
from rbr_b200 import Context, RbrError

pytestmark = pytest.mark.gpu

LOG2_TABLE = 14  # 16384 entries per level: levels 0-1 dense, 2-15 hashed


@pytest.fixture(scope="module")
def cctx():
    c = Context(0)
    yield c
    c.close()


def random_records(rng, n, lo=-1.2, hi=1.2):
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    r[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 9] = rng.uniform(0, 1, n)
    r[:, 10:16] = rng.uniform(0, 1, (n, 6))
    return r


def make_cache(ctx, seed, grid_scale=0.5, weight_scale=1.0):
    """A cache with random parameters set through the C ABI, and its oracle twin."""
    info = ctx.cache_create(log2_table_size=LOG2_TABLE, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1), seed=seed)
    rng = np.random.default_rng(seed)
    grid = rng.uniform(-grid_scale, grid_scale, (rc.LEVELS, 1 << LOG2_TABLE, 2)).astype(np.float16).view(np.uint16)
    w = np.zeros(rc.WEIGHTS, np.float32)
    for l in range(5):
        rows, real = (64, 64) if l < 4 else (16, 3)
        lim = weight_scale * np.sqrt(6.0 / (64 + real))
        blk = rng.uniform(-lim, lim, (rows, 64)).astype(np.float32)
        blk[real:] = 0.0
        w[l * 4096:l * 4096 + rows * 64] = blk.reshape(-1)
    mlp = rc.bf16_bits(w)
    ctx.cache_set_params(mlp, grid.reshape(-1))
    oracle = rc.Cache(list(info.resolution), LOG2_TABLE, [-1, -1, -1], [1, 1, 1], grid, mlp)
    return oracle, rng


def test_cache_configuration_matches_oracle(cctx):
    info = cctx.cache_create(log2_table_size=LOG2_TABLE, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1))
    assert list(info.resolution) == rc.resolutions(16, 2048)
    assert info.dense_levels == rc.dense_mask(rc.resolutions(16, 2048), 1 << LOG2_TABLE)
    assert info.table_size == 1 << LOG2_TABLE and info.optimiser_steps == 0


def test_params_round_trip(cctx):
    oracle, _ = make_cache(cctx, 1)
    m, g = cctx.cache_get_params(grid=True)
    assert np.array_equal(m, oracle.mlp_bits) and np.array_equal(g, oracle.grid_bits.reshape(-1))


@pytest.mark.parametrize("n", [1, 127, 128, 1000])
def test_encoding_bit_exact(cctx, n):
    oracle, rng = make_cache(cctx, 2)
    recs = random_records(rng, n)
    gpu = cctx.cache_encode(recs)
    ref = rc.encode(oracle, recs)
    assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32)), np.argwhere(gpu != ref)[:5]


@pytest.mark.parametrize("n", [1, 129, 2000])
def test_forward_matches_oracle(cctx, n):
    """Tolerance: the oracle accumulates in float64, the tensor cores in FP32; a hidden
    activation that lies on a BF16 rounding boundary can round the other way (one BF16 ulp,
    2^-8 relative). Outputs agree to 1e-2 of their scale, the median to 1e-4."""
    oracle, rng = make_cache(cctx, 3)
    recs = random_records(rng, n)
    gpu = cctx.cache_infer(recs)
    ref = rc.infer(oracle, recs)
    scale = max(1e-3, float(np.abs(ref).max()))
    err = np.abs(gpu - ref) / scale
    assert err.max() < 1e-2, err.max()
    assert np.median(err) < 1e-4, np.median(err)


@pytest.mark.parametrize("n", [300, 4096])
def test_gradients_match_oracle(cctx, n):
    """Weight and hash-grid gradients of one batch against the oracle's float64 backward pass
    with the same BF16 rounding points: relative Frobenius error below 1e-2 per matrix and
    for the grid; the loss to 1e-3."""
    oracle, rng = make_cache(cctx, 4)
    recs = random_records(rng, n)
    targets = rng.uniform(0.0, 2.0, (n, 3)).astype(np.float32)
    loss = cctx.cache_train(recs, targets, apply=False)
    gm, gg = cctx.cache_grads()
    ref_loss, dW, ref_gg = rc.gradients(oracle, recs, targets)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    gpu_dW = rc.split_weights(gm)
    for l in range(5):
        rel = np.linalg.norm(gpu_dW[l] - dW[l]) / max(1e-30, np.linalg.norm(dW[l]))
        assert rel < 1e-2, (l, rel)
    assert np.all(gpu_dW[4][3:] == 0.0)
    ref_gg = ref_gg.reshape(-1)
    rel = np.linalg.norm(gg - ref_gg) / np.linalg.norm(ref_gg)
    assert rel < 1e-2, rel
    # entries the batch did not touch stay exactly zero
    assert np.all(gg[ref_gg == 0.0] == 0.0)


def test_adam_step_matches_oracle(cctx):
    """One optimiser step: the GPU's new BF16 weights and FP16 grid entries equal the oracle's
    float32 Adam applied to the same gradients, except where a gradient is so close to zero
    that its sign differs between the two (atomic) gradient sums."""
    oracle, rng = make_cache(cctx, 5)
    recs = random_records(rng, 2048)
    targets = rng.uniform(0.0, 2.0, (2048, 3)).astype(np.float32)
    cctx.cache_train(recs, targets, apply=False)
    gm, gg = cctx.cache_grads()
    cctx.cache_train(recs, targets, apply=True)
    m_new, g_new = cctx.cache_get_params(grid=True)
    assert cctx.cache_info().optimiser_steps == 1
    p0 = rc.bf16_value(oracle.mlp_bits)
    p1, _, _ = rc.adam(p0, np.zeros_like(p0), np.zeros_like(p0), gm, 1e-2, 0.9, 0.99, 1e-15, 1)
    ref_m = rc.bf16_bits(p1)
    assert np.mean(m_new == ref_m) > 0.999
    grid0 = oracle.grid.reshape(-1, 2)
    g2 = gg.reshape(-1, 2)
    active = np.any(g2 != 0.0, axis=1, keepdims=True) & np.ones((1, 2), bool)
    pg, _, _ = rc.adam(grid0, np.zeros_like(grid0), np.zeros_like(grid0), g2, 1e-2, 0.9, 0.99, 1e-15, 1, active=active)
    ref_g = pg.astype(np.float16).view(np.uint16).reshape(-1)
    assert np.mean(g_new == ref_g) > 0.999
    assert np.array_equal(g_new[~active.reshape(-1)], oracle.grid_bits.reshape(-1)[~active.reshape(-1)])


def test_training_lowers_loss(cctx):
    """Online training on a smooth radiance-like field: the relative L2 loss falls by more than
    10x within 300 steps of 4096 samples."""
    cctx.cache_create(log2_table_size=LOG2_TABLE, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1), seed=7)
    rng = np.random.default_rng(7)

    def field(r):
        p, d = r[:, 0:3], r[:, 3:6]
        base = 0.6 + 0.4 * np.sin(3 * p[:, 0]) * np.cos(2 * p[:, 1]) + 0.2 * p[:, 2]
        return np.stack([base * (1 + 0.3 * d[:, 2]), base * r[:, 10], 0.5 * base + 0.2 * d[:, 0] ** 2], 1).clip(0.01)

    losses = []
    for step in range(300):
        recs = random_records(rng, 4096, -1.0, 1.0)
        losses.append(cctx.cache_train(recs, field(recs).astype(np.float32), apply=True))
    assert np.isfinite(losses).all()
    early, late = np.mean(losses[:5]), np.mean(losses[-20:])
    assert late < early / 10, (early, late)
    recs = random_records(rng, 4096, -1.0, 1.0)
    pred = cctx.cache_infer(recs)
    t = field(recs)
    rel = np.mean((pred - t) ** 2 / (t ** 2 + 1e-2))
    assert rel < 0.05, rel


@pytest.mark.parametrize("groups", [2, 4])
def test_grouped_inference_equals_one_tile_per_cta(cctx, groups):
    """cache.infer_groups: several 128-sample tiles in flight per CTA compute each tile with the
    same MMA sequence and epilogue as one tile per CTA, so the predictions are the same bits;
    a ragged last tile and more tiles than the grid holds at once are covered."""
    _, rng = make_cache(cctx, 7)
    recs = random_records(rng, 5000)
    cctx.set_param("cache.infer_groups", 1)
    want = cctx.cache_infer(recs)
    cctx.set_param("cache.infer_groups", groups)
    try:
        got = cctx.cache_infer(recs)
    finally:
        cctx.set_param("cache.infer_groups", 1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_eight_warp_inference_equals_four_warp(cctx):
    """cache.infer_warps 8: two threads per sample row (hash levels 0-7, and levels 8-15 with the
    other inputs; the epilogues split by accumulator column half) feed the same operands to the
    same MMA sequence as four warps, so the predictions are the same bits; a ragged last tile
    and more tiles than the grid holds at once are covered."""
    _, rng = make_cache(cctx, 11)
    recs = random_records(rng, 150_000)
    cctx.set_param("cache.infer_warps", 4)
    want = cctx.cache_infer(recs)
    cctx.set_param("cache.infer_warps", 8)
    try:
        got = cctx.cache_infer(recs)
    finally:
        cctx.set_param("cache.infer_warps", 4)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    with pytest.raises(RbrError):
        cctx.set_param("cache.infer_warps", 6)


def test_spatially_sorted_inference_equals_given_order(cctx):
    """cache.sort_queries 1: the queries are served in the order of their cells (a counting sort
    on a 32^3 grid, many queries sharing a cell); each query's prediction is the same bits."""
    _, rng = make_cache(cctx, 13)
    recs = random_records(rng, 120_000)
    recs[:20_000, 0:3] = recs[0, 0:3]  # a sixth of them in one cell
    cctx.set_param("cache.sort_queries", 0)
    want = cctx.cache_infer(recs)
    cctx.set_param("cache.sort_queries", 1)
    try:
        got = cctx.cache_infer(recs)
    finally:
        cctx.set_param("cache.sort_queries", 0)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
