"""The product's kNN against the reference's own GPU kNN (cudaKDTree builder +
cct query from src/KNN_GWN.cu, built into oracle/_ref/ by oracle/ref_knn.mk)."""
import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref_knn.so")


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF):
        pytest.skip("reference kNN comparator not built (oracle/ref_knn.mk needs the reference checkout)")
    lib = C.CDLL(REF)
    lib.refknn_build.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    lib.refknn_query.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    return lib


@pytest.mark.parametrize("k", [10, 15])
def test_knn_matches_reference_cukd(ref_lib, k):
    P, _ = D.torus(30000, seed=4)
    Pn, _, _ = D.normalize(P)
    rng = np.random.default_rng(9)
    Q = np.concatenate([Pn[rng.choice(len(Pn), 3000, replace=False)] + rng.normal(0, 0.004, (3000, 3)),
                        rng.uniform(-0.5, 0.5, (1000, 3))]).astype(np.float32)
    tree = torch.from_numpy(Pn.copy()).cuda()
    nrm = torch.zeros_like(tree)
    bounds = np.zeros(6, np.float32)
    assert ref_lib.refknn_build(tree.data_ptr(), nrm.data_ptr(), len(Pn), bounds.ctypes.data) == 0
    Qd = torch.from_numpy(Q).cuda()
    out_ref = torch.empty((len(Q), k), dtype=torch.int32, device="cuda")
    assert ref_lib.refknn_query(tree.data_ptr(), len(Pn), Qd.data_ptr(), len(Q), bounds.ctypes.data,
                                out_ref.data_ptr(), k) == 0
    T = tree.cpu().numpy().astype(np.float64)
    ref_pos = T[out_ref.cpu().numpy()]                     # neighbours, as positions
    Pd = torch.from_numpy(Pn).cuda()
    got = turbo.KnnIndex(Pd).query(Qd, k).cpu().numpy()
    got_pos = Pn.astype(np.float64)[got]
    dr = np.linalg.norm(ref_pos - Q[:, None, :], axis=2)
    dg = np.linalg.norm(got_pos - Q[:, None, :], axis=2)
    # the same k distances in the same order, to FP32 rounding of d^2
    assert np.allclose(np.sort(dr, 1), np.sort(dg, 1), rtol=1e-6, atol=1e-9)
    # the same neighbours (as points) wherever the k-th distance is not a near tie
    same = np.all(np.sort(ref_pos.reshape(len(Q), -1), 1) == np.sort(got_pos.reshape(len(Q), -1), 1), axis=1)
    assert same.mean() > 0.999
