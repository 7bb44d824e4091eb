"""The adjoint (sx_posterior_grad): gradients of the Forward log score lnZ with
respect to every log-space emission and transition score, i.e. the posterior
expected counts.  Checked against

* the oracle's FP64 log-space expected counts (independent recursion);
* the reference's own posterior decoding (decode, src/hmmer/dp.rs:1278-1306):
  the match-emission gradient summed over residues is the column sum of the
  posterior matrix;
* FP64 central finite differences (step 1e-6) of the oracle's log-space
  Forward, through a test-only torch.autograd.Function whose backward is the
  GPU adjoint.

Tolerances: gradients within 1e-3 absolute + 1e-3 relative (f32 accumulation
over L rows); lnZ within 1e-5 relative of the FP64 value.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import sxhmm
from sxhmm import synth
from _workloads import small_config, tiny_text

pytestmark = pytest.mark.gpu
ROWS = ["MM", "MI", "MD", "IM", "II", "DM", "DD"]


@pytest.fixture(scope="module")
def engine():
    e = sxhmm.Engine()
    yield e
    e.close()


@pytest.fixture(scope="module")
def adj_case():
    """Config 3 shapes, shrunk: profiles of M=300, targets of L~400 carrying 0-3 domains."""
    w = synth.make_config(3, scale=1 / 64, scorer=None)
    return w


class Plan7ForwardScore(torch.autograd.Function):
    """lnZ of one (profile, target) pair as a function of the profile's
    log-space scores; backward is the GPU adjoint (test harness only)."""

    @staticmethod
    def forward(ctx, msc, isc, trans, engine, profiles, targets, pi, ti, m):
        lnz, d_msc, d_isc, d_tr = engine.posterior_grad(profiles, targets, [pi], [ti], m)
        ctx.save_for_backward(torch.from_numpy(d_msc[0]).double(), torch.from_numpy(d_isc[0]).double(),
                              torch.from_numpy(d_tr[0]).double())
        return torch.tensor(lnz[0], dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        d_msc, d_isc, d_tr = ctx.saved_tensors
        return g * d_msc, g * d_isc, g * d_tr, None, None, None, None, None, None


def _gpu(engine, text, seqs, pairs, m):
    ps = engine.load_text(text)
    lens = np.array([len(s) for s in seqs], np.int64)
    offs = np.zeros(len(seqs), np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    ts = engine.targets_digital(np.concatenate(seqs).astype(np.uint8), offs, lens)
    pp = [a for a, _ in pairs]
    pt = [b for _, b in pairs]
    return ps, ts, engine.posterior_grad(ps, ts, pp, pt, m)


def _close(got, want, what):
    err = np.abs(got - want)
    bad = err > 1e-3 + 1e-3 * np.abs(want)
    assert not bad.any(), (what, np.argwhere(bad)[:5], got[bad][:5], want[bad][:5])


def test_adjoint_vs_fp64_counts(engine, adj_case):
    w = adj_case
    text = w.hmm_text()
    o = O.Oracle(text=text)
    pairs = w.pairs[:6]
    ps, ts, (lnz, d_msc, d_isc, d_tr) = _gpu(engine, text, w.targets, pairs, 300)
    for q, (pi, ti) in enumerate(pairs):
        ref = o.expected_counts_f64(pi, w.targets[ti])
        assert abs(lnz[q] - ref["lnz"]) <= 1e-5 * max(1.0, abs(ref["lnz"])), (lnz[q], ref["lnz"])
        _close(d_msc[q], ref["d_msc"], "d_msc")
        _close(d_isc[q], ref["d_isc"], "d_isc")
        for r in range(7):
            _close(d_tr[q][r], ref["d_t"][r], ROWS[r])
        _close(d_tr[q][7], ref["d_tbm"], "BM")


def test_adjoint_matches_reference_decoding(engine, adj_case):
    w = adj_case
    text = w.hmm_text()
    o = O.Oracle(text=text)
    pairs = w.pairs[6:10]
    ps, ts, (lnz, d_msc, d_isc, d_tr) = _gpu(engine, text, w.targets, pairs, 300)
    for q, (pi, ti) in enumerate(pairs):
        dec = o.decode(pi, w.targets[ti], multihit=True)  # forward/backward_matrix + decode, Xsc(L, multihit)
        assert abs(lnz[q] - dec["fwd"]) <= 1e-4 * max(1.0, abs(dec["fwd"]))
        col = dec["pm"][1:].sum(0)
        _close(d_msc[q].sum(0), col.astype(np.float64), "sum_x d_msc vs decode pm")
        _close(d_isc[q].sum(0), dec["pi"][1:].sum(0).astype(np.float64), "sum_x d_isc vs decode pi")


def test_adjoint_finite_differences_via_autograd(engine):
    """FP64 central differences of the oracle's log-space Forward vs the
    autograd gradient supplied by the GPU adjoint (tiny model + a synthetic one)."""
    rng = np.random.default_rng(2)
    prof = synth.sample_profile(rng, 40, "fd40")
    text = synth.profile_text(prof) + tiny_text()
    o = O.Oracle(text=text)
    seq = synth.plant(rng, 120, [synth.emit_homolog(rng, prof)])
    tiny_seq = O.encode("GGMKAGGGGGGMKAGG")
    for pi, d, m in ((0, seq, 40), (1, tiny_seq, 3)):
        ps, ts, _ = _gpu(engine, text, [d], [(pi, 0)], m)
        w1 = m + 1
        msc = torch.zeros(25, w1, dtype=torch.float64, requires_grad=True)
        isc = torch.zeros(25, w1, dtype=torch.float64, requires_grad=True)
        tr = torch.zeros(8, w1, dtype=torch.float64, requires_grad=True)
        lnz = Plan7ForwardScore.apply(msc, isc, tr, engine, ps, ts, pi, 0, m)
        lnz.backward()
        h = 1e-6
        x_first = int(d[0])
        checks = [(1, x_first * w1 + 1, msc.grad[x_first, 1]), (3 + 0, 1, tr.grad[0, 1]),
                  (3 + 2, 1, tr.grad[2, 1]), (10, 1, tr.grad[7, 1]), (10, m, tr.grad[7, m])]
        if m > 3:
            checks += [(3 + 1, m // 2, tr.grad[1, m // 2]), (3 + 6, m // 2, tr.grad[6, m // 2]),
                       (1, int(d[len(d) // 2]) * w1 + m // 2, msc.grad[int(d[len(d) // 2]), m // 2])]
        for kind, idx, g in checks:
            fd = (o.forward_f64(pi, d, True, kind, idx, h) - o.forward_f64(pi, d, True, kind, idx, -h)) / (2 * h)
            assert abs(float(g) - fd) <= 1e-3 + 1e-3 * abs(fd), (pi, kind, idx, float(g), fd)


def test_adjoint_out_arrays_reused(engine, adj_case):
    """Gradients written into caller-provided (reused) arrays equal a fresh
    call's; arrays of the wrong shape are refused."""
    w = adj_case
    pairs = w.pairs[:4]
    ps, ts, fresh = _gpu(engine, w.hmm_text(), w.targets, pairs, 300)
    out = tuple(np.full_like(a, np.nan) for a in fresh)
    pp, pt = [a for a, _ in pairs], [b for _, b in pairs]
    engine.posterior_grad(ps, ts, pp, pt, 300, out=out)
    for a, b in zip(fresh, out):
        assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        engine.posterior_grad(ps, ts, pp, pt, 300, out=(out[0], out[1][:, :24], out[2], out[3]))
