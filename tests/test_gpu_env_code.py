"""GPU test of the 32-value environment code (the MLP's environment features,
env_encode_kernel) against a numpy restatement computed from the same packed
rounded-box records (bcc_pack_envs): primitive counts per kind, the signed
distance from 8 fixed anchor points to the nearest primitive of each kind, and
the mean centre and extent.  Counts must agree exactly; distances and means
within 2e-5 (FP32 sums in a different order on the device)."""
import numpy as np
import pytest

from bcc import EnvSet, workload
from bcc.workload import make_capsules, make_cuboids, make_spheres

from test_host import pack

pytestmark = pytest.mark.gpu

ANCHORS = np.array([[0.35 if a & 1 else -0.35, 0.35 if a & 2 else -0.35, 0.8 if a & 4 else 0.3]
                    for a in range(8)])


def env_code_restated(rec, off):
    """Code [N, 32] from packed records [P, 20] and offsets [N + 1] (FP64)."""
    N = len(off) - 1
    code = np.zeros((N, 32))
    for i in range(N):
        r = rec[off[i]:off[i + 1]].astype(np.float64)
        c = code[i]
        rho = r[:, 3]
        hsum = r[:, 7] + r[:, 11] + r[:, 15]
        kind = np.where(rho > 0, np.where(hsum > 0, 1, 0), 2)
        for k in range(3):
            c[k] = np.count_nonzero(kind == k) / 64.0
        c[3] = len(r) / 64.0
        best = np.full((8, 3), 1.5)
        if len(r):
            d = ANCHORS[:, None, :] - r[None, :, 0:3]            # [8, P, 3]
            e2 = np.zeros(d.shape[:2])
            for ax in range(3):
                A = r[:, 4 + 4 * ax:7 + 4 * ax]
                h = r[:, 7 + 4 * ax]
                e = np.maximum(np.abs(np.einsum("apj,pj->ap", d, A)) - h, 0.0)
                e2 += e * e
            dist = np.sqrt(e2) - rho                            # [8, P]
            for k in range(3):
                m = kind == k
                if m.any():
                    best[:, k] = np.minimum(best[:, k], dist[:, m].min(1))
            c[28:31] = r[:, 0:3].mean(0)
            c[31] = (rho + hsum).mean()
        c[4:28] = np.clip(best, -0.5, 1.5).reshape(-1)
    return code


def special_envs():
    rng = np.random.default_rng(3)
    c = rng.uniform(-0.6, 0.6, (6, 3))
    return EnvSet.from_lists([
        {},
        {"spheres": make_spheres(c[:3], [0.1, 0.05, 0.2])},
        {"cuboids": make_cuboids(c[:4], rng.uniform(-3, 3, (4, 3)), rng.uniform(0.02, 0.3, (4, 3)))},
        {"capsules": make_capsules(c[:2], rng.uniform(-3, 3, (2, 3)), np.full(2, 0.05), np.full(2, 0.4))},
        {"spheres": make_spheres(np.array([[0.35, 0.35, 0.8]]), [0.1])},  # anchor inside: distance < 0
        {"spheres": make_spheres(np.array([[5.0, 5.0, 5.0]]), [0.1])},    # beyond the clamp
    ])


@pytest.mark.parametrize("case", ["uneven", "multi_fetch", "special"])
def test_env_code_matches_restatement(checker, case):
    envs = special_envs() if case == "special" else workload.gen_envs(case, 40, seed=17)
    st, rec, off = pack(envs)
    assert st == 0
    checker.upload(envs)
    got = checker.env_code()
    want = env_code_restated(rec, off)
    assert got.shape == (envs.num_envs, 32)
    np.testing.assert_array_equal(got[:, :4], want[:, :4].astype(np.float32))
    np.testing.assert_allclose(got[:, 4:], want[:, 4:], rtol=0, atol=2e-5)
    if case == "special":
        assert got[0, 4:28].tolist() == [1.5] * 24            # empty: no primitive of any kind
        assert got[4, 4 + 7 * 3 + 0] < 0                       # anchor 7 lies inside the sphere
        assert got[5, 4:28].max() == 1.5 and got[5, 4] == 1.5  # clamped
