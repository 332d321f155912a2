"""The reconstruction server on the GPU: every request's image equals the
one SensaRecon gives alone, bit for bit, whatever runs beside it (requests
of other sizes on other streams, cached matrices shared by concurrent
requests of one protocol)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def templates():
    from monalisa_b200 import serving, workloads

    tps = workloads.serving_templates(scale=0.05)
    tps = [tps[0], tps[1], tps[3], tps[4]]  # two 2-D and two 3-D protocols
    for k, tp in enumerate(tps):
        tp["y"] = serving.simulate_data(tp, seed=k)
    return tps


def _alone(tp, nCGD):
    import monalisa_b200 as mb
    import torch

    Gu, Gut = mb.bmTraj2SparseMat(tp["t"], tp["ve"], tp["N_u"], np.ones(tp["imDim"]))
    rec = mb.SensaRecon(Gu, Gut, tp["C"], tp["n_u"])
    y = torch.from_numpy(tp["y"]).cuda()
    ve = torch.from_numpy(np.ascontiguousarray(tp["ve"], np.float32)).cuda()
    x = torch.zeros(int(np.prod(tp["n_u"])), dtype=torch.complex64, device="cuda")
    rec.run_dev(y, ve, x, nIter=1, nCGD=nCGD)
    out = x.cpu().numpy()
    rec.plan.close()
    return out


def test_results_do_not_depend_on_the_mix(templates):
    from monalisa_b200 import serving

    nCGD = 8
    alone = [_alone(tp, nCGD) for tp in templates]
    server = serving.ReconServer(workers=4)
    arrivals = np.zeros(12)  # all at once: maximal overlap
    tmpl = np.array([0, 2, 1, 3, 0, 0, 2, 3, 1, 2, 0, 3])
    reqs = serving.run_poisson(server, templates, arrivals, tmpl, nCGD=nCGD)
    server.close()
    for r, k in zip(reqs, tmpl):
        assert r.error is None, r.error
        assert np.array_equal(r.x, alone[k]), (r.rid, k)
    st = serving.latency_stats(reqs)
    assert st["n"] == 12 and st["p99_ms"] >= st["p50_ms"] > 0
