"""The planner's cost model on the GPU: CUDA forward/backward kernels against
the float64 CPU oracle, training, and what the trained model gains over the
fixed plan rule on classes it was not trained on."""
import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rs():
    import rsgpu

    return rsgpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    assert t.cuda.is_available()
    return t


def rand_data(seed, n):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, M.F)).astype(np.float32)
    t = rng.uniform(5, 11, (n, M.P)).astype(np.float32)
    mask = rng.integers(0, 2, (n, M.P)).astype(np.uint8)
    mask[:, 0] = 1
    return x, t, mask


@pytest.mark.parametrize("n", [1, 37, 1000])
def test_cuda_gradients_match_oracle(rs, torch, n):
    w = M.init(3).astype(np.float32)
    x, t, mask = rand_data(n, n)
    loss, g = rs.Tuner.gradients(w, x, t, mask)
    ref_loss, ref_g = M.loss_and_grad(w.astype(np.float64), x, t, mask)
    # fp32 kernels against the float64 restatement
    assert abs(loss - ref_loss) <= 1e-5 + 1e-4 * abs(ref_loss)
    err = np.abs(g - ref_g)
    assert np.all(err <= 1e-5 + 1e-3 * np.abs(ref_g)), float(err.max())


def test_cuda_forward_matches_oracle(rs, torch):
    w = M.init(9).astype(np.float32)
    rs.Tuner.set_params(w)
    x, _, _ = rand_data(2, 300)
    y = rs.Tuner.predict(x)
    ref = M.forward(w.astype(np.float64), x)
    assert np.allclose(y, ref, rtol=1e-4, atol=1e-4)


def test_training_fits_and_is_deterministic(rs, torch):
    # Targets from a random teacher network: the student must fit them.
    teacher = M.init(11, scale=2.0)
    x, _, mask = rand_data(4, 400)
    y = (M.forward(teacher, x) + 8.0).astype(np.float32)
    l0 = float(((y - 0.0) ** 2 * mask).sum() / mask.sum())
    loss = rs.Tuner.train(x, y, mask, epochs=1500, lr=3e-3, seed=5)
    assert loss < 0.05 * l0 and loss < 0.5, (loss, l0)
    w1 = rs.Tuner.get_params()
    _, g = M.loss_and_grad(w1.astype(np.float64), x, y, mask)
    loss2 = rs.Tuner.train(x, y, mask, epochs=1500, lr=3e-3, seed=5)
    assert loss2 == loss and np.array_equal(rs.Tuner.get_params(), w1)


def fixed_plan(feat, measured):
    """The fixed rule of the planner (batch.cu mix_default_plan): classic ->
    K1 tile 0 (8 KiB items) from 8 KiB shards up; Leopard -> the FFT, largest
    tile whose work rows fit 96 KiB (transforms of <= 16 lanes run in
    registers, where the tile does not matter: any measured FFT plan)."""
    if feat[0] > 0.5:
        return (0, 0) if (0, 0) in measured else (0, 1)
    ffts = sorted(p for p in measured if p[0] == 1)
    k = round(2 ** (feat[3] * 16))
    m = round(2 ** (feat[4] * 16))
    mp = 1 << (m - 1).bit_length()
    n = 1 << (mp + k - 1).bit_length()
    rows = n if feat[7] > 0.5 else 2 * mp
    reg = (n if feat[7] > 0.5 else mp) <= 16
    if reg:
        return ffts[0]
    length = 2 ** (feat[5] * 10 + 12)
    t = 1
    while t < 3 and rows * (64 << (t + 1)) <= 96 * 1024 and (64 << (t + 1)) <= length:
        t += 1
    return (1, t) if (1, t) in measured else ffts[-1]


def _op(rs, codec, op, length, e=0, seed=0):
    k, m = codec.data_shard_count(), codec.parity_shard_count()
    present = None
    if op == "reconstruct":
        rng = np.random.default_rng(seed)
        present = np.ones(k + m, np.uint8)
        present[rng.choice(k + m, size=e, replace=False)] = 0
    return dict(codec=codec, op=op, shards=[1] * (k + m), shard_len=length, present=present)


def test_tuner_table_planner_and_model_gain(rs, torch, tmp_path):
    T = rs.Tuner
    T.clear()
    codecs = {
        ("classic", 10, 4): rs.ReedSolomon(10, 4),
        ("classic", 4, 2): rs.ReedSolomon(4, 2),
        ("leopard_gf8", 32, 16): rs.ReedSolomon(32, 16, rs.CodecOptions(codec_family="leopard_gf8")),
        ("leopard_gf8", 128, 64): rs.ReedSolomon(128, 64, rs.CodecOptions(codec_family="leopard_gf8")),
    }

    def classes(lengths, e_fracs, seed):
        out = []
        for (fam, k, m), c in codecs.items():
            for L in lengths:
                out.append(_op(rs, c, "encode", L))
                out.append(_op(rs, c, "verify", L))
                for i, f in enumerate(e_fracs):
                    out.append(_op(rs, c, "reconstruct", L, max(1, int(round(f * m))), seed + i))
        return out

    train_ops = classes([16384, 262144, 1 << 20], [0.25, 1.0], 1)
    held_ops = classes([65536, 4 << 20], [0.5], 7)
    n_train = T.tune(train_ops, target_bytes=96 << 20, repeats=2)
    assert n_train > 0 and T.table_size() == n_train
    # Every tuned class has a measured best plan.
    for op in train_ops:
        assert T.lookup(op) is not None
    # Save / load round trip.
    path = str(tmp_path / "plans.txt")
    T.save(path)
    n_samples = len(T.samples())
    T.clear()
    assert T.table_size() == 0
    T.load(path)
    assert T.table_size() == n_train and len(T.samples()) == n_samples
    # Train the model on the tuner's own measurements (GPU kernels).
    loss = T.train_from_tuner(epochs=3000, lr=3e-3, seed=1)
    assert T.model_ready() and loss < 1.0, loss
    # Held-out classes (lengths and erasure counts the model never saw):
    # measure them now to know the truth, then score the model's picks and
    # the fixed rule's picks against it.
    before = {tuple(f): None for f, _, _ in T.samples()}
    T.tune(held_ops, target_bytes=96 << 20, repeats=2)
    truth = {}
    for f, plan, g in T.samples():
        if tuple(f) in before:
            continue
        truth.setdefault(tuple(f), {})[plan] = g
    assert truth
    feats = np.array([k for k in truth], np.float32)
    pred = T.predict(feats)
    model_ratio, fixed_ratio = [], []
    for i, key in enumerate(truth):
        meas = truth[key]
        best = max(meas.values())
        valid = [j for j, p in enumerate(rs.MODEL_PLAN_ORDER) if p in meas]
        pick = rs.MODEL_PLAN_ORDER[max(valid, key=lambda j: pred[i, j])]
        model_ratio.append(meas[pick] / best)
        fixed_ratio.append(meas[fixed_plan(key, meas)] / best)
    gain = float(np.mean(model_ratio)) / float(np.mean(fixed_ratio))
    print(f"held-out classes {len(truth)}: model {np.mean(model_ratio):.3f} of best, fixed "
          f"{np.mean(fixed_ratio):.3f} of best, gain {gain:.2f}x")
    assert np.mean(model_ratio) >= np.mean(fixed_ratio)
    assert np.mean(model_ratio) > 0.8
