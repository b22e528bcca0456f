"""GPU tests of the bead dynamics that stand in for OpenMM (include/lbm_b200_md.h): forces against a numpy brute-force
evaluation (bonds excluded from the pair force, minimum image), with the cell list and the brute-force path, and the
leapfrog step."""
import numpy as np
import pytest

import lbm_b200

pytestmark = pytest.mark.gpu


def numpy_forces(pos, box, bonds, k, r0, pair, sigma, eps, cutoff):
    n = len(pos)
    f = np.zeros_like(pos)
    bonded = set()
    for i, j in bonds:
        d = pos[i] - pos[j]
        d -= box*np.round(d/box)
        r = np.sqrt(d.dot(d))
        fb = -k*(r - r0)/r*d
        f[i] += fb
        f[j] -= fb
        bonded.add((min(i, j), max(i, j)))
    rc = 2**(1/6)*sigma if pair == 'wca' else cutoff
    for i in range(n):
        d = pos[i] - pos
        d -= box*np.round(d/box)
        r2 = (d*d).sum(axis=1)
        for j in np.nonzero((r2 < rc*rc) & (r2 > 0))[0]:
            if (min(i, j), max(i, j)) in bonded:
                continue
            s6 = (sigma*sigma/r2[j])**3
            f[i] += 24*eps*s6*(2*s6 - 1)/r2[j]*d[j]
    return f


@pytest.mark.parametrize('pair,box,chains,length', [('wca', 6.0, 4, 25), ('wca', 3.0, 2, 6), ('lj', 11.0, 4, 25),
                                                    ('lj', 4.0, 2, 10)])
def test_forces_match_numpy(pair, box, chains, length):
    """Boxes of 5 and more cells per axis use the cell list, the others the brute-force pass."""
    import torch
    pos, bonds = lbm_b200.random_walk_chains(chains, length, (box, box, box), seed=3)
    pos = pos + np.random.default_rng(1).normal(scale=0.05, size=pos.shape)
    masses = np.ones(len(pos))
    md = lbm_b200.BeadDynamics(masses, (box, box, box), bonds, 5.0, 1.0, pair, 1.0, 0.7, 2.5)
    p = torch.tensor(pos, device='cuda', dtype=torch.float64)
    f = torch.zeros_like(p)
    md.compute_forces(p, f)
    torch.cuda.synchronize()
    expected = numpy_forces(pos, np.array([box]*3), bonds, 5.0, 1.0, pair, 1.0, 0.7, 2.5)
    assert abs(f.cpu().numpy() - expected).max() <= 1e-10*max(1.0, abs(expected).max())
    # Newton's third law: the total force vanishes.
    assert abs(f.sum(dim=0).cpu().numpy()).max() < 1e-9


def test_leapfrog():
    import torch
    masses = np.array([1.0, 2.0, 4.0])
    md = lbm_b200.BeadDynamics(masses, (10.0, 10.0, 10.0), np.zeros((0, 2), dtype=np.int32), 0.0, 1.0, 'none')
    x = torch.tensor([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]], device='cuda', dtype=torch.float64)
    v = torch.tensor([[0.1, 0.0, 0.0], [0.0, 0.2, 0.0], [0.0, 0.0, 0.3]], device='cuda', dtype=torch.float64)
    f = torch.tensor([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], device='cuda', dtype=torch.float64)
    x0, v0 = x.cpu().numpy(), v.cpu().numpy()
    md.integrate(0.5, x, v, f)
    torch.cuda.synchronize()
    v1 = v0 + 0.5*f.cpu().numpy()/masses[:, None]
    assert np.allclose(v.cpu().numpy(), v1, rtol=0, atol=1e-15)
    assert np.allclose(x.cpu().numpy(), x0 + 0.5*v1, rtol=0, atol=1e-15)
    assert abs(md.twice_kinetic(v) - (masses[:, None]*v1*v1).sum()) < 1e-14
