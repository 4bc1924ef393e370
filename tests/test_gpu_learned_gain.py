"""What the shipped learned initialiser gains over the Gauss map it
replaces: on held-out procedural shapes (seeds outside the training range)
its initial leaf normals agree in orientation with the shapes' true normals
more often.  The DWG iterations it saves (none measured on these shapes) are
reported by the benchmark, not asserted here."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import datasets as D, turbo  # noqa: E402
from dwg_b200.train_init import DEFAULT_WEIGHTS  # noqa: E402

pytestmark = pytest.mark.gpu


def agreement(normals, truth):
    return float(((normals * truth).sum(1) > 0).mean())


def test_learned_start_orients_better_than_gauss_map(dwg_lib):
    shapes = {"torus": D.torus(60000, seed=2024),
              "sq12": D.superquadric_union(60000, seed=20001),
              "sq3": D.superquadric_union(60000, k=3, outlier_frac=0.0, noise=0.003, seed=20777)}
    model = turbo.LearnedNormalInit(DEFAULT_WEIGHTS)
    gains = {}
    for name, (P, N) in shapes.items():
        Pn, _, _ = D.normalize(P)
        Pd = torch.from_numpy(np.ascontiguousarray(Pn, np.float32)).cuda()
        d = turbo.TurboDWG(Pd, None, grid_reso=32, final_reso=32, total_iter=0)
        leaves = torch.from_numpy(d.get("leaf_pos")).cuda()
        gauss = d.get("leaf_nrm")
        d.close()
        nb = turbo.KnnIndex(Pd).query(leaves, 1).cpu().numpy()[:, 0]
        truth = N[nb]
        learned = model.init_normals(leaves).cpu().numpy()
        assert np.allclose(np.linalg.norm(learned, axis=1), 1.0, atol=1e-5)
        a_g, a_l = agreement(gauss, truth), agreement(learned, truth)
        gains[name] = (a_g, a_l)
        assert a_l > a_g, (name, a_g, a_l)
    mean_gain = np.mean([l - g for g, l in gains.values()])
    assert mean_gain >= 0.03, gains
