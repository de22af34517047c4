"""The adjoint kernel against finite differences, on a B200.

* In the packed inputs: the gradient of sum(Jbar J) along random directions of each group of
  inputs, against central differences (Richardson-extrapolated) of the (strict) CUDA solve
  itself — the solve is checked
  against the oracle elsewhere, so this checks the adjoint alone; frozen devices included (their
  gradient runs back through the pre-bias solve).
* In the 14 log-parameters of the adjoint workload (`jaxdd_b200.fitting`): autograd through
  `records` and the adjoint against central differences with step 1e-6 (the reference's protocol,
  test_solver.py:1903-1934), and against the oracle's curves differenced the same way for one
  device (the oracle rebuilds the device from its input texts on the same grid structure).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200 import adjoint as adj  # noqa: E402
from jaxdd_b200 import fitting  # noqa: E402
from jaxdd_b200.batch import prepare  # noqa: E402
from jaxdd_b200.workloads import drawn_devices  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

V = np.round(np.linspace(-0.2, 1.2, 8), 10)
S, C, I = _lib.S, _lib.C, _lib.I

GROUPS = {
    "mobilities": [("S", S["MUN"]), ("S", S["MUP"])],
    "spacing": [("S", S["H"]), ("S", S["DX"])],
    "poisson": [("S", S["FACL"]), ("S", S["FACM"]), ("S", S["FACU"]), ("S", S["DOP"])],
    "rows": [("S", S["FAC"]), ("S", S["SP"]), ("S", S["SC"])],
    "offsets": [("S", S["OFFN"]), ("S", S["OFFP"])],
    "recombination": [("S", S["KD"]), ("S", S["NI2"]), ("S", S["NT"]), ("S", S["CNT"]),
                      ("S", S["CPT"]), ("S", S["NT0"]), ("S", S["PT0"]), ("S", S["G"])],
    "contacts": [("C", C["V0"]), ("C", C["VL"]), ("C", C["LNNL"]), ("C", C["LNPL"]),
                 ("C", C["LNNR"]), ("C", C["LNPR"])],
    "scalars": [("C", C["L"]), ("C", C["HSUM"]), ("C", C["GFRAC"]), ("C", C["VPRE"]),
                ("C", _lib.DD_NS_BASE), ("C", _lib.DD_NS_BASE + 1)],
    "interfaces": [("I", I["NT"]), ("I", I["IW"])],
}


@pytest.fixture(scope="module")
def setup():
    devs = drawn_devices(4, NP=100)
    batch = prepare(devs)
    p = adj.plan(batch, V, strict=True)
    cuda = torch.device("cuda")
    rec = tuple(torch.from_numpy(batch[k]).to(cuda) for k in ("stat", "scal", "iface"))
    J, ok, its, ckpt = adj.solve_states(p, *rec)
    rng = np.random.default_rng(3)
    Jbar = torch.from_numpy(rng.uniform(-1, 1, p.nflat) / batch["J_scale"].max()).to(cuda)
    grads = adj.adjoint(p, *rec, ok, ckpt, Jbar)
    return batch, p, rec, J, ok, Jbar, grads


def _direction(rec, group, rng):
    """A random relative perturbation of one group of inputs (zero where the input is)."""
    d = [torch.zeros_like(t) for t in rec]
    for kind, f in group:
        i = "SCI".index(kind)
        t = rec[i]
        sl = (slice(None), f) if kind == "S" else ((f,) if kind == "C" else (slice(None), f))
        base = t[sl]
        r = torch.from_numpy(rng.choice([-1.0, 1.0], size=tuple(base.shape))).to(t.device)
        d[i][sl] = base * r
    return d


@pytest.mark.parametrize("group", list(GROUPS))
def test_input_gradients_match_differences_of_the_solve(setup, group):
    batch, p, rec, J, ok, Jbar, grads = setup
    rng = np.random.default_rng(len(group) * 7 + 1)
    d = _direction(rec, GROUPS[group], rng)
    lin = sum(float((g * di).sum()) for g, di in zip(grads, d))
    # the group's fields one by one: their contributions can cancel in the sum
    parts = 0.0
    for kind, f in GROUPS[group]:
        i = "SCI".index(kind)
        sl = (slice(None), f) if kind in "SI" else (f,)
        parts += abs(float((grads[i][sl] * d[i][sl]).sum()))

    def central(eps):
        vals = []
        for s in (1, -1):
            pert = tuple((t + s * eps * di).contiguous() for t, di in zip(rec, d))
            Jp, okp, _, _ = adj.solve_states(p, *pert)
            assert torch.equal(okp, ok)
            vals.append(float((Jbar * torch.where(ok > 0, Jp, torch.zeros_like(Jp))).sum()))
        return (vals[0] - vals[1]) / (2 * eps)

    # Richardson's extrapolation of two central differences: the Poisson stencils move the
    # solution so strongly that a single difference at 1e-6 keeps a 1e-3 truncation error
    fd = (4 * central(5e-7) - central(1e-6)) / 3
    # the difference's own floor: the solve's round-off in sum(Jbar J) over the step
    mag = float((Jbar.abs() * J.abs()).sum())
    assert abs(lin - fd) <= 2e-4 * max(abs(fd), abs(lin)) + 1e-5 * parts + 1e-6 * mag, (
        group, lin, fd, parts)


@pytest.fixture(scope="module")
def fit_case():
    texts = [fitting.fit_texts(k, NP=120) for k in range(4)]
    st = fitting.Structure(texts)
    Vs = np.round(np.linspace(-0.2, 1.2, 9), 10)
    p = adj.plan(st.batch, Vs, strict=True)
    th0 = torch.tensor(st.theta0, dtype=torch.float64, device=st.device)
    with torch.no_grad():
        Jt, okt, _ = adj.curves(*fitting.records(torch.tensor(
            fitting.target_theta(st.theta0), dtype=torch.float64, device=st.device), st), p)
    scale = torch.tensor(st.batch["J_scale"], device=st.device)
    target = (adj.per_device(p, Jt), adj.per_device(p, okt))
    assert float(target[1].float().mean()) > 0.9
    return st, p, th0, target, scale


def _loss(st, p, theta, target, scale):
    J, ok, _ = adj.curves(*fitting.records(theta, st), p)
    both = adj.per_device(p, ok) * target[1]
    return fitting.misfit(adj.per_device(p, J), both, target[0], scale)


def test_parameter_gradients_match_central_differences(fit_case):
    st, p, th0, target, scale = fit_case
    th = th0.clone().requires_grad_(True)
    loss = _loss(st, p, th, target, scale)
    loss.backward()
    g = th.grad.cpu().numpy()
    h = 1e-6
    fd = np.zeros(th0.shape[1])
    with torch.no_grad():
        for j in range(th0.shape[1]):
            e = torch.zeros_like(th0)
            e[:, j] = h  # every device at once: the loss is a sum over devices
            lp = float(_loss(st, p, th0 + e, target, scale))
            lm = float(_loss(st, p, th0 - e, target, scale))
            fd[j] = (lp - lm) / (2 * h)
    total = g.sum(0)
    for j, name in enumerate(fitting.NAMES):
        assert abs(total[j] - fd[j]) <= 1e-4 * np.abs(total).max() + 1e-3 * abs(fd[j]), (
            name, total[j], fd[j])


@pytest.mark.parametrize("k", [0, 1])
def test_one_device_against_the_oracle(fit_case, k):
    """Device 0 (ions frozen after its pre-bias) and device 1 (free ions): the GPU's gradient of
    one curve's weighted sum in all 14 parameters against the oracle's curves differenced in each
    (central, step 1e-6 and 5e-7, Richardson-extrapolated)."""
    from jaxdd_b200.device import build_device
    from jaxdd_b200.simss_input import setup_from_texts
    from oracle import dd
    st, p, th0, target, scale = fit_case
    Vs = p.v.cpu().numpy()[:9]
    w = np.random.default_rng(11).uniform(-1, 1, 9) / st.batch["J_scale"][k]
    th = th0.clone().requires_grad_(True)
    J, ok, _ = adj.curves(*fitting.records(th, st), p)
    Jd = adj.per_device(p, J)
    (Jd[k] * torch.from_numpy(w).to(Jd.device)).sum().backward()
    g = th.grad[k].cpu().numpy()

    def oracle(theta):
        dev = build_device(setup_from_texts(fitting.texts_with(st.texts[k], theta)),
                           layout=st.layouts[k])
        Jo, oko, _ = dd.solve_batch(dd.prepare([dev]), Vs, strict=True)
        assert oko.all()
        return float(np.sum(w * Jo[0]))

    def central(j, h):
        e = np.zeros(14)
        e[j] = h
        return (oracle(st.theta0[k] + e) - oracle(st.theta0[k] - e)) / (2 * h)

    fds = np.array([(4 * central(j, 5e-7) - central(j, 1e-6)) / 3 for j in range(14)])
    top = np.abs(fds).max()
    for j, name in enumerate(fitting.NAMES):
        assert abs(g[j] - fds[j]) <= 1e-4 * abs(fds[j]) + 1e-7 * top, (name, g[j], fds[j])
