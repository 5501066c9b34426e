"""Generates tests/golden/known_answers.npz: closed-form known answers for the
CIC gather/deposit, the leapfrog push and the cell binning of PSuM's
electrostatic path.

These do not come from any implementation under test.  Each case is small
enough to check by hand:
  * CIC weights of linear_interp on simple_grid (src/field/simple_grid.hpp:316-349,
    simple_interpolation.hpp:34-54): w = prod_a (1-t_a or t_a), t = frac((p-lo)/dx);
  * the gradient of the bilinear/trilinear interpolant of a linear potential
    phi = g . x is g exactly, so one leapfrog step in it is closed form
    (application/benchmark/TSI/main.cpp:59-75);
  * deposit of a few particles = sum of their CIC weights (field_interp.hpp:66-75);
  * binning keys c2i(nC(p)) with nC = trunc((p-lo)/dx) for lo <= p < hi,
    counts, exclusive offsets and the stable permutation
    (grid_mapped_device_vector.hpp:47-87).
Run: python tests/golden/make_golden.py
"""
import os

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.npz")


def cic_2d(p, lo, dx, cells):
    """indices and weights (support order: bit 0 = last axis) on the node lattice."""
    u = [(p[a] - lo[a]) / dx[a] for a in range(2)]
    b = [int(np.floor(u[a])) for a in range(2)]
    t = [u[a] - b[a] for a in range(2)]
    idx, w = [], []
    for i in range(4):
        bi, bj = (i >> 1) & 1, i & 1
        ni = (b[0] + bi) % (cells[0] + 1)
        nj = (b[1] + bj) % (cells[1] + 1)
        idx.append(ni * (cells[1] + 1) + nj)
        w.append((t[0] if bi else 1 - t[0]) * (t[1] if bj else 1 - t[1]))
    return idx, w


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    # --- 2-D CIC on [0,1]^2 with 8x8 cells (dx = 1/8 exactly)
    cells = (8, 8)
    lo, dx = (0.0, 0.0), (0.125, 0.125)
    pts = np.array([[0.3, 0.55], [0.0, 0.0], [0.5, 0.5], [0.999, 0.001], [0.1875, 0.8125]])
    I, W = [], []
    for p in pts:
        i, w = cic_2d(p, lo, dx, cells)
        I.append(i)
        W.append(w)
    out["cic2_points"] = pts
    out["cic2_idx"] = np.array(I, np.int64)
    out["cic2_w"] = np.array(W)

    # --- leapfrog in a linear potential phi = gx*x + gy*y on a Dirichlet 16x16 box [0,16)^2
    gx, gy = 0.03, -0.02
    n = 64
    pos = rng.uniform(2.0, 14.0, size=(2, n))
    vel = rng.normal(0.0, 0.5, size=(3, n))
    qm, dt = -1.0, 0.1
    E = np.array([-gx, -gy])
    v_new = vel.copy()
    v_new[0] += E[0] * qm * dt
    v_new[1] += E[1] * qm * dt
    p_new = pos + v_new[:2] * dt
    xs = np.arange(17.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    out["push_phi"] = (gx * X + gy * Y).ravel()
    out["push_pos0"] = pos
    out["push_vel0"] = vel
    out["push_pos1"] = p_new
    out["push_vel1"] = v_new
    out["push_qm_dt"] = np.array([qm, dt])

    # --- deposit of 3 particles on the 8x8 grid above, weight 1 each
    dep_pts = np.array([[0.3, 0.55], [0.31, 0.56], [0.9, 0.1]])
    rho = np.zeros(81)
    for p in dep_pts:
        i, w = cic_2d(p, lo, dx, cells)
        for k in range(4):
            rho[i[k]] += w[k]
    out["dep_points"] = dep_pts
    out["dep_rho"] = rho

    # --- binning of 12 particles on [0,4)x[0,3) with 4x3 cells (dx = 1)
    bp = np.array([[0.5, 0.5], [3.9, 2.9], [1.2, 0.1], [0.5, 0.7], [4.0, 1.0], [-0.1, 1.0],
                   [1.99, 2.0], [0.0, 0.0], [2.5, 1.5], [0.2, 0.9], [3.0, 3.0], [1.5, 0.5]]).T
    keys, counts = [], np.zeros(12, np.uint64)
    for i in range(bp.shape[1]):
        x, y = bp[0, i], bp[1, i]
        if 0.0 <= x < 4.0 and 0.0 <= y < 3.0:
            k = int(x) * 3 + int(y)
            keys.append(k)
            counts[k] += 1
        else:
            keys.append(-1)
    offsets = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint64)
    perm = [i for k in range(12) for i in range(bp.shape[1]) if keys[i] == k]
    out["bin_pos"] = bp
    out["bin_keys"] = np.array(keys, np.int64)
    out["bin_counts"] = counts
    out["bin_offsets"] = offsets
    out["bin_perm"] = np.array(perm, np.uint64)
    np.savez(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
