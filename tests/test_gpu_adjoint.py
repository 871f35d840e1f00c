"""exchange_halo and its adjoint as a differentiable pair.

A shifted Lennard-Jones energy (epsilon = sigma = 1, rc = 2.5) at density 0.8
over N = 262,144 uniform particles is evaluated from the owned positions and
the ghost positions that exchange_halo makes of them.  A torch.autograd.Function
(test-side) wraps the halo: forward refreshes the ghosts from the owned
positions along the plan, backward scatter-adds the ghost cotangents to their
owners with dsx_grid_halo_backward.  The autograd gradient is checked against
central finite differences (h = 1e-6) on 64 seeded coordinates, on a 2x2x2
virtual grid (ghosts carry the cross-subdomain pairs) and at 1x1x1 (no
ghosts, as in the reference at one rank: the energy there uses minimum
images).  That the backward equals reverse_halo on identical cotangents is
test_gpu_parity.py::test_halo_backward_is_reverse_halo.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 262_144
DENSITY = 0.8
L = (N / DENSITY) ** (1.0 / 3.0)
RC = 2.5
HALO = 2.8
H = 1e-6


class DeviceArray:
    """A raw device pointer as a CUDA-array-interface object for torch.as_tensor."""

    def __init__(self, ptr, n, typestr="<f8"):
        self.__cuda_array_interface__ = dict(shape=(n,), typestr=typestr, data=(ptr, False),
                                             version=3, strides=None)


def lj(r2):
    """Shifted LJ pair energy for squared distances r2 (r < rc masked by the caller)."""
    inv6 = 1.0 / r2 ** 3
    rc6 = 1.0 / RC ** 6
    return 4.0 * (inv6 * inv6 - inv6) - 4.0 * (rc6 * rc6 - rc6)


class Halo:
    """The grid's owned/ghost position arrays as torch views, and the halo pair."""

    def __init__(self, torch, grid):
        self.torch, self.grid = torch, grid
        v = grid.view()
        self.n = int(v.particles)
        o, g = grid.all_counts()
        self.counts_owned, self.counts_ghost = o, g
        self.G = int(g.sum())
        self.owned = [torch.as_tensor(DeviceArray(v.base[a] + 8 * int(v.owned_offset), self.n),
                                      device="cuda") for a in range(3)]
        self.ghost = [torch.as_tensor(DeviceArray(v.base[a] + 8 * int(v.ghost_offset), self.G),
                                      device="cuda") for a in range(3)] if self.G else None
        self.gid_owned = torch.as_tensor(DeviceArray(v.base[12] + 4 * int(v.owned_offset), self.n, "<i4"),
                                         device="cuda").clone()
        self.gid_ghost = (torch.as_tensor(DeviceArray(v.base[12] + 4 * int(v.ghost_offset), self.G, "<i4"),
                                          device="cuda").clone() if self.G else None)

    def refresh(self, x):
        """Owned positions x (3, n) into the grid, ghosts refreshed along the plan."""
        torch = self.torch
        for a in range(3):
            self.owned[a].copy_(x[a])
        torch.cuda.synchronize()
        self.grid.exchange_halo(positions_only=True)
        torch.cuda.synchronize()
        if not self.G:
            return x.new_zeros((3, 0))
        return torch.stack([t.clone() for t in self.ghost])

    def function(self):
        halo = self

        class HaloExchange(halo.torch.autograd.Function):
            @staticmethod
            def forward(ctx, x):
                return halo.refresh(x.detach())

            @staticmethod
            def backward(ctx, cot):
                grad = cot.new_zeros((3, halo.n))
                if halo.G:
                    cot = cot.contiguous()
                    halo.torch.cuda.synchronize()
                    halo.grid.halo_backward(cot, grad)
                    halo.torch.cuda.synchronize()
                return grad

        return HaloExchange.apply


def pair_lists(halo, x, xg, periodic_box):
    """Pairs within rc + 0.1 of the current positions: (i, j, weight, kind)
    with kind 0 owned-owned and 1 owned-ghost (j indexes the ghosts).  Each
    subdomain pairs its owned particles with its owned particles and ghosts;
    an owned-ghost pair is seen from both sides, so it weighs 1/2."""
    from scipy.spatial import cKDTree
    xo = x.detach().cpu().numpy().T
    xgh = xg.detach().cpu().numpy().T if halo.G else np.zeros((0, 3))
    o, g = halo.counts_owned, halo.counts_ghost
    ob, gb = np.concatenate([[0], np.cumsum(o)]), np.concatenate([[0], np.cumsum(g)])
    ii, jj, ww, kk = [], [], [], []
    for s in range(len(o)):
        own = xo[ob[s]:ob[s + 1]]
        pts = np.concatenate([own, xgh[gb[s]:gb[s + 1]]])
        if periodic_box:
            tree = cKDTree(np.mod(pts, L), boxsize=L)
        else:
            tree = cKDTree(pts)
        p = tree.query_pairs(RC + 0.1, output_type="ndarray")
        if not len(p):
            continue
        a, b = np.minimum(p[:, 0], p[:, 1]), np.maximum(p[:, 0], p[:, 1])
        no = len(own)
        oo = b < no
        og = (a < no) & (b >= no)
        ii.append(ob[s] + a[oo]); jj.append(ob[s] + b[oo]); ww.append(np.ones(oo.sum())); kk.append(np.zeros(oo.sum(), int))
        ii.append(ob[s] + a[og]); jj.append(gb[s] + b[og] - no); ww.append(np.full(og.sum(), 0.5)); kk.append(np.ones(og.sum(), int))
    return [np.concatenate(v) for v in (ii, jj, ww, kk)]


def energy_terms(torch, x, xg, pairs, min_image):
    i, j, w, k = pairs
    dev = x.device
    i_t = torch.as_tensor(i, device=dev)
    j_t = torch.as_tensor(j, device=dev)
    w_t = torch.as_tensor(w, device=dev, dtype=torch.float64)
    k_t = torch.as_tensor(k, device=dev)
    xi = x[:, i_t]
    xj = torch.where(k_t.bool(), xg[:, j_t.clamp(max=max(xg.shape[1] - 1, 0))] if xg.shape[1] else xi,
                     x[:, j_t.clamp(max=x.shape[1] - 1)])
    d = xi - xj
    if min_image:
        d = d - L * torch.round(d / L)
    r2 = (d * d).sum(0)
    e = torch.where(r2 < RC * RC, lj(r2), torch.zeros_like(r2))
    return w_t * e


@pytest.mark.parametrize("dims", [(2, 2, 2), (1, 1, 1)], ids=["2x2x2", "1x1x1"])
def test_lj_gradient_through_halo_adjoint(cuda, dims):
    import torch

    import dsdecompx_b200 as dsx
    P = int(np.prod(dims))
    rng = np.random.default_rng(404)
    pos = rng.uniform(0.0, L, size=(N, 3))
    data = {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(),
            "global_id": np.arange(N, dtype=np.int32), "mass": np.ones(N)}
    empty = {k: v[:0] for k, v in data.items()}
    grid = dsx.VirtualGrid(P, dims, "manual", (0.0, 0.0, 0.0), (L, L, L), halo_width=HALO,
                           particles=N, ghost_capacity=2 * N)
    try:
        grid.upload([data] + [empty] * (P - 1))
        grid.migrate()
        grid.exchange_halo(rebuild=True)
        torch.cuda.synchronize()
        halo = Halo(torch, grid)
        assert (halo.G > 0) == (P > 1)
        exchange = halo.function()
        x0 = torch.stack([t.clone() for t in halo.owned])          # (3, n) as owned now
        xg0 = halo.refresh(x0)
        pairs = pair_lists(halo, x0, xg0, periodic_box=(P == 1))
        min_image = P == 1

        # autograd gradient of the total energy
        x = x0.clone().requires_grad_(True)
        e = energy_terms(torch, x, exchange(x), pairs, min_image).sum()
        e.backward()
        grad = x.grad.detach()

        # 64 seeded coordinates: owned particles with ghost images first (their
        # gradient flows through the adjoint), nearest neighbour >= 0.6 apart
        from scipy.spatial import cKDTree
        xo = x0.cpu().numpy().T
        nearest = cKDTree(np.mod(xo, L), boxsize=L).query(np.mod(xo, L), k=2)[0][:, 1]
        gid_o = halo.gid_owned.cpu().numpy()
        imaged = np.zeros(halo.n, bool)
        if halo.G:
            order = np.argsort(gid_o)
            imaged[order[np.searchsorted(gid_o[order], np.unique(halo.gid_ghost.cpu().numpy()))]] = True
        good = nearest >= 0.6
        pool_img = np.flatnonzero(good & imaged)
        pool_int = np.flatnonzero(good & ~imaged)
        n_img = 48 if P > 1 else 0
        picks = np.concatenate([rng.choice(pool_img, n_img, replace=False),
                                rng.choice(pool_int, 64 - n_img, replace=False)])
        axes = rng.integers(0, 3, size=64)

        i_all, j_all, _, k_all = pairs
        gid_g = halo.gid_ghost.cpu().numpy() if halo.G else np.zeros(0, np.int32)
        for p, a in zip(picks, axes):
            images = np.flatnonzero(gid_g == gid_o[p])
            sel = (i_all == p) | ((k_all == 0) & (j_all == p)) | ((k_all == 1) & np.isin(j_all, images))
            local = [v[sel] for v in pairs]
            vals = []
            for sgn in (1.0, -1.0):
                xp = x0.clone()
                xp[a, p] += sgn * H
                xgp = halo.refresh(xp)
                vals.append(energy_terms(torch, xp, xgp, local, min_image).sum().item())
            fd = (vals[0] - vals[1]) / (2.0 * H)
            g = grad[a, p].item()
            assert abs(fd - g) <= 1e-6 * max(1.0, abs(g)), (p, a, fd, g)
        halo.refresh(x0)
    finally:
        grid.close()
