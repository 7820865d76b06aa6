"""Learned table selector, host side: the fp64 MLP oracle against finite
differences, the parameter file format, and the oracle's restatement of the
learned form's passes (no GPU)."""
import numpy as np
import pytest

import oracle
import oracle.mlp as M
import bzip2gpu_b200.selector as S
import bzip2gpu_b200.workloads as W


def _groups(seed=3, n=300000):
    st, info = oracle.compress_block(W.small_markov(n, seed=seed))
    return M.groups_of_stream(st["rle2"]), st, info


def test_oracle_gradients_match_finite_differences():
    gs, _, _ = _groups()
    gs = gs[:64]
    c, n = M.features(gs)
    rng = np.random.default_rng(5)
    P = S.init_params(7).astype(np.float64)
    P[M.B1_:M.W2_] = rng.normal(0, 0.1, M.HID)
    P[M.B2_:M.W3_] = rng.normal(0, 0.1, M.HID)
    P[M.B3_:M.B3_ + M.OUT] = rng.normal(0, 0.1, M.OUT)
    y = rng.integers(0, 6, gs.shape[0])
    _, _, g = M.loss_grads(P, c, n, y, emulate=False)

    def loss(Q):
        return M.loss_grads(Q, c, n, y, emulate=False)[0] / gs.shape[0]

    # coordinates of every tensor, padding excluded
    picks = [M.W1_ + 3 * M.IN_PAD + 1, M.W1_ + 200 * M.IN_PAD + 0, M.B1_ + 17, M.W2_ + 1000,
             M.W2_ + 40000, M.B2_ + 3, M.W3_ + 2 * M.HID + 9, M.W3_ + 5 * M.HID + 100,
             M.B3_ + 0, M.B3_ + 4]
    h = 1e-5
    for k in picks:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd = (loss(Pp) - loss(Pm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])
    # padding carries no gradient
    assert np.all(g[M.W1_:M.B1_].reshape(M.HID, M.IN_PAD)[:, M.IN:] == 0)
    assert np.all(g[M.W3_:M.B3_].reshape(M.OUT_PAD, M.HID)[M.OUT:] == 0)
    assert np.all(g[M.B3_ + M.OUT:] == 0)


def test_oracle_features_are_group_histograms():
    gs, st, _ = _groups()
    c, n = M.features(gs)
    syms = st["rle2"]
    assert n.sum() == syms.size and np.all(n[:-1] == 50)
    assert np.array_equal(c.sum(0)[: M.IN], np.bincount(syms, minlength=M.IN)[: M.IN])


def test_parameter_file_round_trip(tmp_path):
    P = S.init_params(11)
    P[S.OFF_B1:S.OFF_W2] = np.linspace(-1, 1, S.HID)
    f = tmp_path / "w.bin"
    S.save(P, f)
    Q = S.load(f)
    assert f.stat().st_size == 8 + 2 * (256 * 258 + 256 * 256 + 6 * 256) + 4 * (256 + 256 + 6)
    # weights are stored as bf16, biases exactly
    assert np.array_equal(Q[S.OFF_B1:S.OFF_W2], P[S.OFF_B1:S.OFF_W2])
    W = np.concatenate([P[S.OFF_W1:S.OFF_B1], P[S.OFF_W2:S.OFF_B2], P[S.OFF_W3:S.OFF_B3]])
    Wq = np.concatenate([Q[S.OFF_W1:S.OFF_B1], Q[S.OFF_W2:S.OFF_B2], Q[S.OFF_W3:S.OFF_B3]])
    assert np.array_equal(Wq, M.bf16(W).astype(np.float32))
    # padding stays zero
    assert np.all(Q[S.OFF_W1:S.OFF_B1].reshape(S.HID, S.IN_PAD)[:, S.IN:] == 0)
    with pytest.raises(ValueError):
        (tmp_path / "bad.bin").write_bytes(b"nope")
        S.load(tmp_path / "bad.bin")


@pytest.mark.parametrize("seed", [3, 8])
def test_refine_from_plain_choice_reproduces_plain_tables(seed):
    # the learned form's passes, started from the plain selector's final
    # choice with no exact pass, rebuild exactly the plain tables
    _, st, info = _groups(seed, 900000)
    ln, code, sel = oracle.huffman_refine(st["rle2"], info.n_in_use, st["sel"], 0)
    a = info.n_in_use + 2
    assert np.array_equal(sel, st["sel"])
    assert np.array_equal(ln[:, :a], st["len"][:, :a])
    assert np.array_equal(code[:, :a], st["code"][:, :a])


def test_coded_bits_counts_payload_selectors_tables():
    _, st, info = _groups(4, 200000)
    syms, sel, ln = st["rle2"], st["sel"], st["len"]
    bits = oracle.coded_bits(syms, sel, info.n_groups, info.n_in_use, ln)
    _, pay = oracle.encode(syms, sel, ln, st["code"])
    smtf = oracle.selector_mtf(sel, info.n_groups)
    a = info.n_in_use + 2
    tables = sum(5 + sum(2 * abs(int(ln[t, v]) - (int(ln[t, v - 1]) if v else int(ln[t, 0]))) + 1
                         for v in range(a)) for t in range(info.n_groups))
    assert bits == pay + int(smtf.sum()) + smtf.size + tables


def test_selector_specs_reach_block_count():
    sp = W.selector_specs(200, 0xB2C3)
    blocks = sum(-(-s.size // (s.level * 100000)) for s in sp)
    assert blocks >= 200 and blocks - max(-(-sp[-1].size // (sp[-1].level * 100000)), 1) < 200
    # the same draws as the config-2 generator with that seed
    assert [(s.size, s.level) for s in sp[:5]] == \
        [(s.size, s.level) for s in W.batch_specs(5, 0xB2C3)]


def test_learned_oracle_judge():
    # the MLP's choice replaced by the plain selector's own final choice:
    # one exact pass keeps (or improves) it, so no fallback; a constant
    # choice (one table for every group) is worse than the plain selector's
    # first two passes, so the block falls back to exactly that selection
    _, st, info = _groups(9, 600000)
    syms = st["rle2"]
    ln, code, sel, ng, fb = oracle.huffman_learned(syms, info.n_in_use, st["sel"])
    assert not fb and ng == 6
    ref = oracle.huffman_refine(syms, info.n_in_use, st["sel"], 1)
    assert np.array_equal(sel, ref[2])
    ln, code, sel, ng, fb = oracle.huffman_learned(syms, info.n_in_use,
                                                   np.zeros_like(st["sel"]))
    assert fb
    pl, pc, ps, png = oracle.huffman_build(syms, info.n_in_use, passes=2)
    assert np.array_equal(sel, ps)
    a = info.n_in_use + 2
    assert np.array_equal(ln[:, :a], pl[:, :a])
    assert np.array_equal(code[:, :a], pc[:, :a])
    # four passes are the reference's selector
    fl, fc, fs, fng = oracle.huffman_build(syms, info.n_in_use)
    assert np.array_equal(fs, st["sel"]) and np.array_equal(fl[:, :a], st["len"][:, :a])
    # fewer than six tables: plain
    _, st2, info2 = _groups(10, 1500)
    assert info2.n_groups < 6
    ln, code, sel, ng, fb = oracle.huffman_learned(st2["rle2"], info2.n_in_use,
                                                   np.zeros(len(st2["sel"]), np.uint8))
    assert not fb and np.array_equal(sel, st2["sel"])
