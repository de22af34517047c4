"""The adjoint workload's parameter map on the CPU: `records` (torch) against the device builder
and the packer it restates, at the reference parameters and at perturbed ones; the parameters'
round trip through the input texts; the target's perturbation."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import _lib, fitting  # noqa: E402
from jaxdd_b200.batch import prepare  # noqa: E402
from jaxdd_b200.device import build_device  # noqa: E402
from jaxdd_b200.simss_input import setup_from_texts  # noqa: E402

TEXTS = [fitting.fit_texts(k, NP=90) for k in range(3)]


def _packed(texts, theta, layouts):
    devs = [build_device(setup_from_texts(fitting.texts_with(t, th)), layout=lay)
            for t, th, lay in zip(texts, theta, layouts)]
    return prepare(devs)


def _compare(got, b):
    for name, g in zip(("stat", "scal", "iface"), got):
        ref = b[name]
        rel = np.abs(g.numpy() - ref) / np.maximum(np.abs(ref), 1e-300)
        if name == "stat":
            # dx: the packer differences the cumulative grid, the map multiplies L h
            dx = rel[:, _lib.S["DX"]]
            rel[:, _lib.S["DX"]] = 0.0
            assert dx.max() < 1e-9
        assert rel.max() < 1e-12, (name, np.argwhere(rel >= 1e-12)[:4])


def test_parameters_round_trip_through_the_texts():
    th = fitting.theta_of(TEXTS[0])
    assert th.shape == (14,) and np.all(np.isfinite(th))
    th2 = th + np.linspace(-0.1, 0.1, 14)
    assert np.allclose(fitting.theta_of(fitting.texts_with(TEXTS[0], th2)), th2, rtol=0,
                       atol=1e-14)
    # both interfaces carry the one density
    t = fitting.texts_with(TEXTS[0], th2)
    assert fitting._get(t["L1.txt"], "N_t_int") == fitting._get(t["L2.txt"], "N_t_int")


def test_records_match_the_builder_and_packer():
    st = fitting.Structure(TEXTS, device="cpu")
    th = torch.tensor(st.theta0, dtype=torch.float64)
    _compare(fitting.records(th, st), st.batch)


def test_records_match_at_perturbed_parameters():
    st = fitting.Structure(TEXTS, device="cpu")
    rng = np.random.default_rng(2)
    theta = st.theta0 + rng.normal(scale=0.05, size=st.theta0.shape)
    W_L, W_R = fitting.flat_band(theta)  # keep the contacts in their gaps
    theta[:, fitting.NAMES.index("W_L")] = np.log(W_L)
    theta[:, fitting.NAMES.index("W_R")] = np.log(W_R)
    got = fitting.records(torch.tensor(theta, dtype=torch.float64), st)
    b = _packed(TEXTS, theta, st.layouts)
    assert np.array_equal(b["lane_of"], st.batch["lane_of"])
    # the current scale (not an input of the residual) is held at the reference parameters
    b["scal"][_lib.C["JSCALE"]] = st.batch["scal"][_lib.C["JSCALE"]]
    _compare(got, b)


def test_records_are_differentiable():
    st = fitting.Structure(TEXTS[:1], device="cpu")
    th = torch.tensor(st.theta0, dtype=torch.float64, requires_grad=True)
    rec0 = [t.detach() for t in fitting.records(th, st)]
    ws = [torch.linspace(0.5, 1.5, t.numel(), dtype=torch.float64).reshape(t.shape)
          / (t.abs() + 1e-300) for t in rec0]  # every entry relative to its own size

    def f(theta):
        return sum((t * w).sum() for t, w in zip(fitting.records(theta, st), ws))

    (g,) = torch.autograd.grad(f(th), th)
    h = 1e-6
    for j in range(14):
        e = torch.zeros_like(th)
        e[0, j] = h
        with torch.no_grad():
            fd = float(f(th + e) - f(th - e)) / (2 * h)
        assert abs(float(g[0, j]) - fd) <= 1e-6 * max(abs(fd), 1.0), (j, float(g[0, j]), fd)


def test_target_perturbation():
    th = np.stack([fitting.theta_of(t) for t in TEXTS])
    tg = fitting.target_theta(th)
    assert np.array_equal(tg, fitting.target_theta(th))
    d = tg - th
    keep = [j for j, n in enumerate(fitting.NAMES) if n not in ("W_L", "W_R")]
    assert 0.05 < np.std(d[:, keep]) < 0.5
    W_L, W_R = fitting.flat_band(tg)
    assert np.allclose(np.exp(tg[:, fitting.NAMES.index("W_L")]), W_L)
    assert np.all((W_L > 2.6) & (W_L < 5.6) & (W_R > 4.0) & (W_R < 7.2))
