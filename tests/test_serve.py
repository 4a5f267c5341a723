"""Serving loop: requests that arrive while others run are admitted between
chunks and step together with them (two lattices at once); each result is
the same as the request run alone through the plain single-case call.
FP32 storage; differences come only from the order of FP64 atomics in force
spreading: final populations relative L2 <= 1e-5, Cd / Cl series rtol 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.serve import Request, Server, make_request, poisson_arrivals, run_alone  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def test_served_results_match_alone():
    rng = np.random.default_rng(11)
    kinds = ["cylinder", "airfoil", "duct", "sphere", "cylinder", "duct"]
    steps = [23, 31, 17, 12, 9, 14]
    reqs = [make_request(i, k, rng, s, scale=0.25) for i, (k, s) in enumerate(zip(kinds, steps))]
    for r, t in zip(reqs, [0.0, 0.0, 0.05, 0.1, 0.15, 0.2]):
        r.arrival = t
    srv = Server(storage="f32", chunk=4)
    stats = srv.run(reqs, keep_f=True)
    srv.close()
    assert stats["requests"] == len(reqs)
    assert stats["p99_latency_s"] >= stats["p50_latency_s"] > 0.0
    assert stats["mlups"] > 0.0
    for r in reqs:
        a = run_alone(r, "f32", keep_f=True)
        assert rel_l2(r.f_final, a.f_final) <= 1e-5, (r.kind, r.rid)
        np.testing.assert_allclose(r.mean_u, a.mean_u, rtol=1e-4, atol=1e-9)
        if r.ib is not None:
            assert r.cd_cl.shape == (r.steps, 2)
            np.testing.assert_allclose(r.cd_cl, a.cd_cl, rtol=1e-4, atol=1e-7)


def test_admission_respects_the_budget():
    """With a budget for about one request, the others wait in the queue and
    are admitted as memory frees up; all still finish."""
    r0 = make_request(0, "cylinder", np.random.default_rng(5), 6, scale=0.25)
    reqs = [Request(i, r0.kind, r0.case, r0.ib, r0.init, 6) for i in range(3)]  # equal footprints
    fp = Server.footprint(r0, "f32")
    srv = Server(storage="f32", chunk=3, hbm_budget=int(1.5 * fp))
    stats = srv.run(reqs)
    srv.close()
    adm = sorted(r.admitted for r in reqs)
    fin = sorted(r.finished for r in reqs)
    assert stats["requests"] == 3
    # never two at once: each later admission happens after an earlier finish
    assert adm[1] >= fin[0] - 1e-9 and adm[2] >= fin[1] - 1e-9


def test_poisson_arrivals_are_seeded():
    a = poisson_arrivals(50, 10.0, np.random.default_rng(3))
    b = poisson_arrivals(50, 10.0, np.random.default_rng(3))
    np.testing.assert_array_equal(a, b)
    assert np.all(np.diff(a) > 0) and abs(a[-1] / 50 - 0.1) < 0.05
