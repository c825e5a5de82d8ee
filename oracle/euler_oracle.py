"""CPU restatement (numpy) of the per-Newton-update path of mfem_euler2d_cpp.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it is imported by
tests/ and by __graft_entry__.smoke(), never by the engine in
mfem_euler2d_cpp_b200/ (which has no CPU fallback).  Every function restates
the reference's algorithm and cites the reference file:line it follows
(paths are relative to the reference project).

Parity is pinned: tests/test_oracle_cpu.py checks every function here against
the golden fixtures in tests/golden/, which were produced by the unmodified
reference sources compiled against an MFEM-subset shim (oracle/Makefile,
oracle/ref_harness.cpp, tests/golden/make_golden.py).

Notation (src/problem.cpp:35-37): q = k+1 points per direction, p = q^2
nodes per cell, m = 4p body unknowns per cell, t = 4q trace unknowns per face,
n = nx*ny cells, nf = 2n faces.  Body vector u[e*m + 4*i + c], node
i = iy*q + ix (x fastest); trace vector l[f*t + 4*j + c] (include/euler.hpp:44-45).
Face f = 2*(iy*nx + ix) + axis; an x-face joins side 1 of its left cell to
side 0 of the cell to its right, a y-face side 3 to side 2 (src/problem.cpp:77-90).
Everything is FP64.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PI = math.pi
EPS = np.finfo(np.float64).eps
TINY = np.finfo(np.float64).tiny


class OracleError(RuntimeError):
    """A failed require() of the reference (include/euler.hpp:19-23); the
    message is the reference's own text."""


def require(cond, msg: str) -> None:
    if not cond:
        raise OracleError(msg)


# ----------------------------------------------------------------------------
# Tables (src/problem.cpp:91-222)
# ----------------------------------------------------------------------------

def gauss_legendre01(q: int):
    """q-point Gauss-Legendre rule on [0, 1] in ascending order (the segment
    rule of order 2q-1 the reference asks MFEM for, src/problem.cpp:131)."""
    t, w = np.polynomial.legendre.leggauss(q)
    return 0.5 * (t + 1.0), 0.5 * w


def lagrange_derivative_matrix(x: np.ndarray) -> np.ndarray:
    """D[a, i] = l_i'(x_a) for the Lagrange basis on nodes x (barycentric form)."""
    q = len(x)
    lam = np.array([1.0 / np.prod([x[i] - x[j] for j in range(q) if j != i]) for i in range(q)])
    D = np.zeros((q, q))
    for a in range(q):
        for i in range(q):
            if i != a:
                D[a, i] = lam[i] / lam[a] / (x[a] - x[i])
        D[a, a] = -D[a].sum()
    return D


def lagrange_values(x: np.ndarray, s: float) -> np.ndarray:
    """l_i(s) for the Lagrange basis on nodes x (product formula)."""
    q = len(x)
    out = np.ones(q)
    for i in range(q):
        for j in range(q):
            if j != i:
                out[i] *= (s - x[j]) / (x[i] - x[j])
    return out


@dataclass
class Tables:
    """Collocated Qk tables on the reference square (src/problem.cpp:91-200)."""
    q: int
    w: np.ndarray          # (p,) volume weights, node order
    ew: np.ndarray         # (q,) edge weights
    ex: np.ndarray         # (q,) edge points
    mass: np.ndarray       # (p,) diagonal of the collocated mass matrix
    inv_mass: np.ndarray   # (p,)
    tdx: np.ndarray        # (q, q) tensor_dx(a, i), already divided by hx
    tdy: np.ndarray        # (q, q) tensor_dy(a, j), already divided by hy
    fv: np.ndarray         # (4, q, p) face restriction (side, face point, node)

    @property
    def p(self) -> int:
        return self.q * self.q


def make_tables(k: int, hx: float, hy: float) -> Tables:
    """Restates the table construction of src/problem.cpp:91-200 for the
    collocated Gauss-Legendre Qk element: volume weights are tensor products of
    the edge rule, the mass matrix is diagonal (collocation), derivative and
    face tables drop entries below 1e-14 (problem.cpp:109-111, 159)."""
    q = k + 1
    x, w1 = gauss_legendre01(q)
    w = np.outer(w1, w1).reshape(-1)           # node iy*q+ix -> w1[iy]*w1[ix]
    D = lagrange_derivative_matrix(x)
    D = np.where(np.abs(D) < 1e-14, 0.0, D)
    l0, l1 = lagrange_values(x, 0.0), lagrange_values(x, 1.0)
    l0 = np.where(np.abs(l0) < 1e-14, 0.0, l0)
    l1 = np.where(np.abs(l1) < 1e-14, 0.0, l1)
    fv = np.zeros((4, q, q * q))
    for j in range(q):                         # face point j
        for iy in range(q):
            for ix in range(q):
                i = iy * q + ix
                fv[0, j, i] = l0[ix] * (iy == j)   # x = 0, y = x_j
                fv[1, j, i] = l1[ix] * (iy == j)   # x = 1
                fv[2, j, i] = l0[iy] * (ix == j)   # y = 0, x = x_j
                fv[3, j, i] = l1[iy] * (ix == j)   # y = 1
    return Tables(q=q, w=w, ew=w1.copy(), ex=x, mass=w.copy(), inv_mass=1.0 / w,
                  tdx=D / hx, tdy=D / hy, fv=fv)


def tables_from_fixture(z) -> Tables:
    """Tables as the reference computed them (tests/golden/units_*.npz)."""
    k = int(z["k"])
    q = k + 1
    p = q * q
    tn = np.asarray(z["tensor_node"])
    require(np.array_equal(tn, np.arange(p)), "GL quadrature/nodal ordering mismatch")
    return Tables(q=q, w=np.array(z["w"]), ew=np.array(z["ew"]), ex=gauss_legendre01(q)[0],
                  mass=np.array(z["mass"]), inv_mass=np.array(z["inv_mass"]),
                  tdx=np.array(z["tensor_dx"]).reshape(q, q), tdy=np.array(z["tensor_dy"]).reshape(q, q),
                  fv=np.array(z["fv"]).reshape(4, q, p))


# ----------------------------------------------------------------------------
# Physics (src/physics.cpp:5-93), vectorised over leading axes
# ----------------------------------------------------------------------------

class Gas:
    def __init__(self, gamma: float = 3.0):
        self.gamma = gamma
        self.gm1 = gamma - 1.0

    def pressure(self, u):                                   # physics.cpp:5-7
        return self.gm1 * (u[..., 3] - 0.5 * (u[..., 1] ** 2 + u[..., 2] ** 2) / u[..., 0])

    def positive(self, u):                                   # physics.cpp:8-11
        with np.errstate(all="ignore"):
            fin = np.all(np.isfinite(u), axis=-1)
            return fin & (u[..., 0] > 1e-13) & (self.pressure(u) > 1e-13)

    def flux(self, u, axis: int):                            # physics.cpp:12-17
        vn = u[..., axis + 1] / u[..., 0]
        p = self.pressure(u)
        f = np.stack([u[..., axis + 1], u[..., 1] * vn, u[..., 2] * vn, (u[..., 3] + p) * vn], axis=-1)
        f[..., axis + 1] += p
        return f

    def jacobian(self, u, axis: int):                        # physics.cpp:18-39; J[..., c, d]
        inv = 1.0 / u[..., 0]
        vx, vy = u[..., 1] * inv, u[..., 2] * inv
        vn = u[..., axis + 1] * inv
        H = u[..., 3] + self.pressure(u)
        g = self.gm1
        dp = np.stack([0.5 * g * (vx * vx + vy * vy), -g * vx, -g * vy, np.full_like(vx, g)], axis=-1)
        dv = np.zeros(u.shape)
        dv[..., 0] = -vn * inv
        dv[..., axis + 1] = inv
        J = np.zeros(u.shape[:-1] + (4, 4))
        J[..., 0, axis + 1] = 1.0
        for d in range(2):
            J[..., d + 1, :] = u[..., d + 1, None] * dv
            if d == axis:
                J[..., d + 1, :] += dp
            J[..., d + 1, d + 1] += vn
        J[..., 3, :] = vn[..., None] * dp + H[..., None] * dv
        J[..., 3, 3] += vn
        return J

    def speeds(self, l, r, axis: int, safety: float):        # physics.cpp:40-63
        fin = np.all(np.isfinite(l), axis=-1) & np.all(np.isfinite(r), axis=-1)
        require(np.all(fin & (l[..., 0] > 1e-13) & (r[..., 0] > 1e-13)),
                "Nonpositive old face state; refine mesh")
        pl, pr = self.pressure(l), self.pressure(r)
        require(np.all((pl > 1e-13) & (pr > 1e-13)), "Nonpositive old face state; refine mesh")
        il, ir = 1.0 / l[..., 0], 1.0 / r[..., 0]
        sl, sr = np.sqrt(l[..., 0]), np.sqrt(r[..., 0])
        v = [(sl * l[..., d + 1] * il + sr * r[..., d + 1] * ir) / (sl + sr) for d in range(2)]
        h = (sl * (l[..., 3] + pl) * il + sr * (r[..., 3] + pr) * ir) / (sl + sr)
        c2 = self.gm1 * (h - 0.5 * (v[0] * v[0] + v[1] * v[1]))
        require(np.all(c2 > 0), "Invalid Roe sound speed")
        ct = np.sqrt(c2)
        cl = np.sqrt(self.gamma * pl * il)
        cr = np.sqrt(self.gamma * pr * ir)
        a = safety * np.maximum(np.maximum(0.0, cl - l[..., axis + 1] * il), ct - v[axis])
        b = safety * np.maximum(np.maximum(0.0, cr + r[..., axis + 1] * ir), ct + v[axis])
        return a, b

    def exact(self, x, y, time: float, alpha: float):        # physics.cpp:64-93
        drift, amplitude = (3.0 - self.gamma) / 2.0, (self.gamma + 1.0) / 4.0
        require(time >= 0 and time * PI * amplitude < 1, "Exact solution requires T < 4/((gamma+1)*pi)")
        phase = math.cos(alpha) * np.asarray(x, float) + math.sin(alpha) * np.asarray(y, float)
        phase = phase - 2 * np.floor((phase + 1) / 2)
        phase = phase - time * drift
        phase = phase - 2 * np.floor((phase + 1) / 2)
        lo, hi, z = phase - time * amplitude, phase + time * amplitude, phase.copy()
        done = np.zeros(z.shape, bool)
        for _ in range(80):
            res = z + time * amplitude * np.sin(PI * z) - phase
            done |= np.abs(res) < 2e-15
            hi = np.where(~done & (res > 0), z, hi)
            lo = np.where(~done & ~(res > 0), z, lo)
            qn = z - res / (1 + time * amplitude * PI * np.cos(PI * z))
            znew = np.where((qn >= lo) & (qn <= hi), qn, 0.5 * (lo + hi))
            z = np.where(done, z, znew)
            if done.all():
                break
        jm = np.sin(PI * z)
        v = 1 + 0.5 * jm
        sound = self.gm1 * (2.0 - jm) / 4.0
        rho = (sound * sound / self.gamma) ** (1.0 / self.gm1)
        pres = rho ** self.gamma
        return np.stack([rho, rho * v * math.cos(alpha), rho * v * math.sin(alpha),
                         pres / self.gm1 + 0.5 * rho * v * v], axis=-1)


# ----------------------------------------------------------------------------
# Problem: residual, Jacobians, condensation (src/problem.cpp, partial.cpp,
# condensation.cpp, operators.cpp)
# ----------------------------------------------------------------------------

# Per cell side s: (is_left, axis); side 1 and 3 are the left cell's sides of
# its own x- and y-face (src/problem.cpp:77-90, 150-156).
SIDE_LEFT = (False, True, False, True)
SIDE_AXIS = (0, 0, 1, 1)


class Problem:
    """Restates euler::Problem (include/euler.hpp:161-230) for the collocated
    Gauss-Legendre discretisation on a periodic Cartesian mesh."""

    def __init__(self, nx: int, ny: int, k: int, alpha_deg: float, safety: float = 1.1,
                 gamma: float = 3.0, tables: Tables | None = None):
        require(nx >= 2 and ny >= 2 and 0 <= k <= 8, "Invalid mesh or degree")
        require(0 < alpha_deg < 90, "Angle must be strictly between 0 and 90 degrees")
        self.nx, self.ny, self.k = nx, ny, k
        self.gas = Gas(gamma)
        self.safety = safety
        self.alpha = alpha_deg * PI / 180                   # problem.cpp:33-36
        self.lx, self.ly = 2 / math.cos(self.alpha), 2 / math.sin(self.alpha)
        self.hx, self.hy = self.lx / nx, self.ly / ny
        self.area = self.hx * self.hy
        self.q = q = k + 1
        self.p = p = q * q
        self.m, self.t = 4 * p, 4 * q
        self.n = n = nx * ny
        self.nf = nf = 2 * n
        self.nu, self.nl = n * self.m, nf * self.t
        self.tab = tables if tables is not None else make_tables(k, self.hx, self.hy)
        tb = self.tab
        I = np.eye(q)
        # Gx[qpt, node], Gy[qpt, node]: collocated derivative tables (problem.cpp:105-111)
        self.Gx = np.kron(I, tb.tdx)
        self.Gy = np.kron(tb.tdy, I)
        # faces (problem.cpp:77-90)
        iy, ix = np.divmod(np.arange(n), nx)
        self.face_l = np.repeat(np.arange(n), 2)
        right_x = iy * nx + (ix + 1) % nx
        right_y = ((iy + 1) % ny) * nx + ix
        self.face_r = np.stack([right_x, right_y], axis=1).reshape(-1)
        self.face_len = np.tile([self.hy, self.hx], n)
        # cell_faces[e, side] (problem.cpp:85-86)
        cf = np.zeros((n, 4), int)
        cf[:, 1] = 2 * np.arange(n)
        cf[:, 3] = 2 * np.arange(n) + 1
        cf[:, 0] = 2 * (iy * nx + (ix - 1) % nx)
        cf[:, 2] = 2 * (((iy - 1) % ny) * nx + ix) + 1
        self.cell_faces = cf
        # dual-norm metrics (problem.cpp:209-222)
        self.cell_metric = np.tile(np.repeat(self.area * tb.mass, 4), n)
        self.trace_metric = (self.face_len[:, None, None] / tb.ew[None, :, None]
                             * np.ones((1, 1, 4))).reshape(-1)
        self.old = np.zeros(self.nu)
        self.dt = 0.0
        self.a = self.b = None

    # -- helpers -------------------------------------------------------------
    def cells(self, u):
        return np.asarray(u, float).reshape(self.n, self.p, 4)

    def side_values(self, u, side: int, cells=None):
        """Eval(u, e, fv[side], q) for all cells (problem.cpp:238-258) -> (n, q, 4)."""
        U = self.cells(u) if cells is None else cells
        return np.einsum("ji,eic->ejc", self.tab.fv[side], U)

    def face_states(self, u):
        """Left/right face-point states per face: (nf, q, 4) each."""
        U = self.cells(u)
        L = np.empty((self.nf, self.q, 4))
        R = np.empty((self.nf, self.q, 4))
        L[0::2] = self.side_values(None, 1, U)
        L[1::2] = self.side_values(None, 3, U)
        R[0::2] = self.side_values(None, 0, U)[self.face_r[0::2]]
        R[1::2] = self.side_values(None, 2, U)[self.face_r[1::2]]
        return L, R

    def _by_axis(self, fn, *arrays):
        """Apply fn(axis, *slices) on the x-faces (even ids) and y-faces (odd)."""
        out0 = fn(0, *[a[0::2] for a in arrays])
        out1 = fn(1, *[a[1::2] for a in arrays])
        if isinstance(out0, tuple):
            res = []
            for o0, o1 in zip(out0, out1):
                o = np.empty((self.nf,) + o0.shape[1:])
                o[0::2], o[1::2] = o0, o1
                res.append(o)
            return tuple(res)
        o = np.empty((self.nf,) + out0.shape[1:])
        o[0::2], o[1::2] = out0, out1
        return o

    def _scatter_faces(self, contrib_l, contrib_r):
        """Add per-face point contributions (nf, q, 4) to the left cell through
        its side restriction and to the right cell through its own
        (problem.cpp:495-505; partial.cpp:113-126)."""
        fv = self.tab.fv
        Y = np.zeros((self.n, self.p, 4))
        ls = np.where(np.arange(self.nf) % 2 == 0, 1, 3)
        rs = ls - 1
        cl = np.einsum("fji,fjc->fic", fv[ls], contrib_l)
        cr = np.einsum("fji,fjc->fic", fv[rs], contrib_r)
        np.add.at(Y, self.face_l, cl)
        np.add.at(Y, self.face_r, cr)
        return Y

    # -- Freeze / WaveRate (problem.cpp:350-384) -----------------------------
    def freeze(self, u, step: float, check_admissible: bool = True):
        if check_admissible:
            require(self.admissible(u), "Old state is inadmissible; refine mesh")
        self.old = np.array(u, float)
        self.dt = step
        L, R = self.face_states(u)
        a, b = self._by_axis(lambda ax, l, r: self.gas.speeds(l, r, ax, self.safety), L, R)
        require(np.all(a + b > 0), "Degenerate HLL speeds")
        self.a, self.b = a, b
        self.inv_sum = 1.0 / (a + b)
        self.lw = b * self.inv_sum
        self.rw = a * self.inv_sum
        self.pen = a * b * self.inv_sum
        return self.wave_rate()

    def wave_rate(self):
        return max(0.0, float(np.max(np.maximum(self.a, self.b)))) / min(self.hx, self.hy)

    # -- CellNorm / Admissible (problem.cpp:259-275, 385-391) ----------------
    def cell_norm(self, r):
        require(len(r) == self.nu, "Cell norm size mismatch")
        return math.sqrt(float(np.sum(self.cell_metric * r * r)))

    def admissible(self, u):
        U = self.cells(u)
        if not np.all(self.gas.positive(U)):
            return False
        for s in range(4):
            if not np.all(self.gas.positive(self.side_values(None, s, U))):
                return False
        return True

    # -- Residual (problem.cpp:445-507) ---------------------------------------
    def residual(self, u):
        tb = self.tab
        U = self.cells(u)
        Fx, Fy = self.gas.flux(U, 0), self.gas.flux(U, 1)
        wF = tb.w[None, :, None]
        R = -self.dt * (np.einsum("qi,eqc->eic", self.Gx, wF * Fx)
                        + np.einsum("qi,eqc->eic", self.Gy, wF * Fy))
        L, Rs = self.face_states(u)
        fl = self._by_axis(lambda ax, s: self.gas.flux(s, ax), L)
        fr = self._by_axis(lambda ax, s: self.gas.flux(s, ax), Rs)
        hl = self.lw[..., None] * fl + self.rw[..., None] * fr + self.pen[..., None] * (L - Rs)
        scale = (self.dt * self.face_len / self.area)[:, None] * tb.ew[None, :]
        R += self._scatter_faces(scale[..., None] * hl, -scale[..., None] * hl)
        R *= tb.inv_mass[None, :, None]
        return R.reshape(-1) + np.asarray(u, float) - self.old

    # -- Partial-assembly DG Jacobian (partial.cpp:31-135) --------------------
    def dg_refresh(self, u):
        U = self.cells(u)
        self._jx = self.gas.jacobian(U, 0)
        self._jy = self.gas.jacobian(U, 1)
        L, R = self.face_states(u)
        JL = self._by_axis(lambda ax, s: self.gas.jacobian(s, ax), L)
        JR = self._by_axis(lambda ax, s: self.gas.jacobian(s, ax), R)
        I4 = np.eye(4)
        self._jl = self.lw[..., None, None] * JL + self.pen[..., None, None] * I4
        self._jr = self.rw[..., None, None] * JR - self.pen[..., None, None] * I4

    def dg_apply(self, x):
        """y = J x at the refreshed state (partial.cpp:62-135)."""
        tb = self.tab
        X = self.cells(x)
        wdt = (self.dt * tb.w)[None, :, None]
        fx = wdt * np.einsum("eqcd,eqd->eqc", self._jx, X)
        fy = wdt * np.einsum("eqcd,eqd->eqc", self._jy, X)
        Y = -(np.einsum("qi,eqc->eic", self.Gx, fx) + np.einsum("qi,eqc->eic", self.Gy, fy))
        L, R = self.face_states(x)
        z = np.einsum("fjcd,fjd->fjc", self._jl, L) + np.einsum("fjcd,fjd->fjc", self._jr, R)
        scale = (self.dt * self.face_len / self.area)[:, None] * tb.ew[None, :]
        Y += self._scatter_faces(scale[..., None] * z, -scale[..., None] * z)
        Y *= tb.inv_mass[None, :, None]
        return Y.reshape(-1) + np.asarray(x, float)

    def volume_blocks(self, u):
        """VolumeJacobianCell for every cell (problem.cpp:519-550): (n, m, m)."""
        tb = self.tab
        U = self.cells(u)
        jx, jy = self.gas.jacobian(U, 0), self.gas.jacobian(U, 1)
        W = (self.dt * tb.w)[:, None]
        A = -(np.einsum("qi,eqcd->eicqd", W * self.Gx, jx) + np.einsum("qi,eqcd->eicqd", W * self.Gy, jy))
        A *= tb.inv_mass[None, :, None, None, None]
        A = A.reshape(self.n, self.m, self.m)
        A += np.eye(self.m)[None]
        return A

    def _face_block(self, side, J, scale):
        """sum_j scale_j inv_mass_i fv[s][j,i] fv[s][j,l] J_j(c,d) as (N, m, m)."""
        tb = self.tab
        f = tb.fv[side]
        B = np.einsum("Nj,ji,jl,Njcd->Nicld", scale, f * tb.inv_mass[None, :], f, J)
        return B.reshape(J.shape[0], self.m, self.m)

    def dg_jacobi_blocks(self, u):
        """PartialDG DiagonalBlocks (partial.cpp:272-297): (n, m, m)."""
        self.dg_refresh(u)
        A = self.volume_blocks(u)
        scale = (self.dt * self.face_len / self.area)[:, None] * self.tab.ew[None, :]
        for f0, ls in ((0, 1), (1, 3)):
            sl = slice(f0, None, 2)
            np.add.at(A, self.face_l[sl], self._face_block(ls, self._jl[sl], scale[sl]))
            np.add.at(A, self.face_r[sl], -self._face_block(ls - 1, self._jr[sl], scale[sl]))
        return A

    # -- HDG condensation (problem.cpp:598-702; condensation.cpp:131-163) ----
    def hdg_cell_pieces(self, u):
        """A_e (n, m, m), C_e (n, 4, q, 4, 4), B scalar lifts (n, 4, q) and D (nl)."""
        tb = self.tab
        A = self.volume_blocks(u)
        U = self.cells(u)
        C = np.empty((self.n, 4, self.q, 4, 4))
        Bs = np.empty((self.n, 4, self.q))
        I4 = np.eye(4)
        for s in range(4):
            left, axis = SIDE_LEFT[s], SIDE_AXIS[s]
            f = self.cell_faces[:, s]
            stab = (self.a if left else self.b)[f]                 # (n, q)
            J = self.gas.jacobian(self.side_values(None, s, U), axis)
            deriv = (1.0 if left else -1.0) * J + stab[..., None, None] * I4
            scale = (self.dt * self.face_len[f] / self.area)[:, None] * tb.ew[None, :]
            A += self._face_block(s, deriv, scale)
            C[:, s] = -tb.ew[None, :, None, None] * deriv
            Bs[:, s] = -scale * stab
        D = np.repeat((tb.ew[None, :] * (self.a + self.b)), 4, axis=1).reshape(-1)
        return A, C, Bs, D

    def lift_dense(self, Bs):
        """FaceCoupling::Dense for the lift B (operators.cpp:119-142): (n, m, 4t)."""
        tb = self.tab
        n, q, p = self.n, self.q, self.p
        B = np.zeros((n, p, 4, 4, q, 4))
        I4 = np.eye(4)
        for s in range(4):
            w = tb.fv[s].T * tb.inv_mass[:, None]                  # (p, q)
            B[:, :, :, s, :, :] = np.einsum("iq,eq,cd->eicqd", w, Bs[:, s], I4)
        return B.reshape(n, self.m, 4 * self.t)

    def restrict(self, Y):
        """Per-cell face restriction of body columns: (n, m, K) -> (n, 4, q, 4, K)."""
        Yc = Y.reshape(self.n, self.p, 4, -1)
        return np.stack([np.einsum("ji,eidk->ejdk", self.tab.fv[s], Yc) for s in range(4)], axis=1)

    def condense(self, u, r):
        """StreamCondense (condensation.cpp:131-148): X, y, rhs, D."""
        A, C, Bs, D = self.hdg_cell_pieces(u)
        B = self.lift_dense(Bs)
        RHS = np.concatenate([B, np.asarray(r, float).reshape(self.n, self.m, 1)], axis=2)
        require(np.all(np.isfinite(A)), "Singular streaming HDG cell factor")
        try:
            XY = np.linalg.solve(A, RHS)                            # row-pivoted LU per cell
        except np.linalg.LinAlgError as exc:
            raise OracleError("Singular streaming HDG cell factor") from exc
        X, y = XY[:, :, :-1], XY[:, :, -1]
        cy = np.einsum("esjcd,esjd->esjc", C, self.restrict(y[..., None])[..., 0])
        rhs = np.zeros(self.nl)
        self._scatter_trace(rhs, cy.reshape(self.n, 4 * self.t))
        self.X, self.y, self.C, self.Bs, self.D = X, y, C, Bs, D
        return X, y, rhs, D

    def trace_ids(self):
        """ids[e] of HybridCell (problem.cpp:648-656): (n, 4t)."""
        return (self.cell_faces[:, :, None] * self.t + np.arange(self.t)[None, None, :]).reshape(self.n, -1)

    def _scatter_trace(self, out, local):
        np.add.at(out, self.trace_ids(), local)

    def schur_apply(self, v):
        """S v = D v - sum_e C_e X_e v[ids_e] (operators.cpp:147-179)."""
        loc = np.asarray(v, float)[self.trace_ids()]               # (n, 4t)
        body = np.einsum("emk,ek->em", self.X, loc)
        cz = np.einsum("esjcd,esjd->esjc", self.C, self.restrict(body[..., None])[..., 0])
        out = self.D * v
        self._scatter_trace(out, -cz.reshape(self.n, 4 * self.t))
        return out

    def schur_jacobi_blocks(self):
        """ElementOperator::DiagonalBlocks on the condensed operator
        (operators.cpp:275-303, Panel operators.cpp:7-26): (nf, t, t)."""
        t = self.t
        blocks = np.zeros((self.nf, t, t))
        idx = np.arange(t)
        blocks[:, idx, idx] = self.D.reshape(self.nf, t)
        RX = self.restrict(self.X)                                  # (n, 4, q, 4, 4t)
        for s in range(4):
            panel = np.einsum("ejcd,ejdk->ejck", self.C[:, s], RX[:, s][..., s * t:(s + 1) * t])
            np.add.at(blocks, self.cell_faces[:, s], -panel.reshape(self.n, t, t))
        return blocks

    def schur_panels(self):
        """All 16 panels C_s R_s X_{:,o} of every cell (FaceCoupling::Panel,
        operators.cpp:7-26): (n, 4, 4, t, t) indexed [cell, s, o]."""
        t = self.t
        RX = self.restrict(self.X)                                  # (n, 4, q, 4, 4t)
        out = np.empty((self.n, 4, 4, t, t))
        for s in range(4):
            full = np.einsum("ejcd,ejdk->ejck", self.C[:, s], RX[:, s]).reshape(self.n, t, 4 * t)
            for o in range(4):
                out[:, s, o] = full[:, :, o * t:(o + 1) * t]
        return out

    def recover(self, lam):
        """du_e = -X_e lam[ids_e] - y_e (condensation.cpp:9-42, 149-163)."""
        loc = np.asarray(lam, float)[self.trace_ids()]
        return (-np.einsum("emk,ek->em", self.X, loc) - self.y).reshape(-1)

    def recovered_residual(self, eps_s):
        """er = -B (eps_S / D) (stepper.cpp:10-26)."""
        scaled = (np.asarray(eps_s, float) / self.D)[self.trace_ids()]
        B = self.lift_dense(self.Bs)
        return (-np.einsum("emk,ek->em", B, scaled)).reshape(-1)

    # -- Integral / Errors / Initial (problem.cpp:329-349, 704-761) -----------
    def _fine_rule(self):
        order = max(24, 2 * self.k + 8)
        xs, ws = gauss_legendre01(order // 2 + 1)
        return xs, ws

    def _fine_shape(self, xs):
        """Basis values at fine points: (nfine, nfine, p) with node iy*q+ix."""
        x = self.tab.ex
        L = np.stack([lagrange_values(x, s) for s in xs])          # (nfine, q)
        return np.einsum("ai,bj->baji", L, L).reshape(len(xs), len(xs), self.p)

    def _cell_origins(self):
        iy, ix = np.divmod(np.arange(self.n), self.nx)
        return -0.5 * self.lx + ix * self.hx, -0.5 * self.ly + iy * self.hy

    def initial(self):
        """L2 projection of the exact wave at t = 0 (problem.cpp:329-349)."""
        xs, ws = self._fine_rule()
        S = self._fine_shape(xs)                                    # (b, a, p): point (x_a, y_b)
        ox, oy = self._cell_origins()
        X = ox[:, None, None] + self.hx * xs[None, None, :]
        Y = oy[:, None, None] + self.hy * xs[None, :, None]
        V = self.gas.exact(np.broadcast_to(X, (self.n, len(xs), len(xs))),
                           np.broadcast_to(Y, (self.n, len(xs), len(xs))), 0.0, self.alpha)
        W = np.outer(ws, ws)
        U = np.einsum("ba,bai,ebac->eic", W, S, V)
        U *= self.tab.inv_mass[None, :, None]
        return U.reshape(-1)

    def integral(self, u):
        U = self.cells(u)
        return self.area * np.einsum("q,eqc->c", self.tab.w, U)

    def errors(self, u, time: float):
        xs, ws = self._fine_rule()
        S = self._fine_shape(xs)
        ox, oy = self._cell_origins()
        X = np.broadcast_to(ox[:, None, None] + self.hx * xs[None, None, :], (self.n, len(xs), len(xs)))
        Y = np.broadcast_to(oy[:, None, None] + self.hy * xs[None, :, None], (self.n, len(xs), len(xs)))
        V = self.gas.exact(X, Y, time, self.alpha)
        Z = np.einsum("bai,eic->ebac", S, self.cells(u))
        W = np.outer(ws, ws)
        return np.sqrt(self.area * np.einsum("ba,ebac->c", W, (Z - V) ** 2))


# ----------------------------------------------------------------------------
# Block ILU(0) (src/block_ilu.cpp:10-124, partial.cpp:140-170, operators.cpp:48-74)
# ----------------------------------------------------------------------------

def solver_graph(pb: Problem, hdg: bool):
    """Problem::SolverGraph (block_ilu.cpp:110-124): cells and their face
    neighbours (DG) or faces sharing a cell (HDG), sorted and unique."""
    if hdg:
        graph = [set() for _ in range(pb.nf)]
        for local in pb.cell_faces:
            for i in local:
                graph[i].update(int(j) for j in local)
    else:
        graph = [{e} for e in range(pb.n)]
        for f in range(pb.nf):
            graph[pb.face_l[f]].add(int(pb.face_r[f]))
            graph[pb.face_r[f]].add(int(pb.face_l[f]))
    return [sorted(g) for g in graph]


class BlockILU0:
    """FixedBlockILU with natural ordering (block_ilu.cpp:10-109): BSR rows
    with sorted columns, the retained ILU(0) products per strictly-lower
    entry, in-place factorisation with pivoted diagonal LU, and the forward
    (unit lower) / backward (upper, diagonal LU solve) apply."""

    def __init__(self, graph, block: int):
        self.rows, self.b = len(graph), block
        self.row, self.col, self.diag = [0], [], []
        for i in range(self.rows):
            for j in sorted(set(graph[i]) | {i}):
                if j == i:
                    self.diag.append(len(self.col))
                self.col.append(j)
            self.row.append(len(self.col))
        self.updates = [[] for _ in self.col]                     # block_ilu.cpp:46-57
        for i in range(self.rows):
            for ik in range(self.row[i], self.diag[i]):
                k = self.col[ik]
                ij, kj = ik + 1, self.diag[k] + 1
                while ij < self.row[i + 1] and kj < self.row[k + 1]:
                    if self.col[ij] < self.col[kj]:
                        ij += 1
                    elif self.col[kj] < self.col[ij]:
                        kj += 1
                    else:
                        self.updates[ik].append((ij, kj))
                        ij += 1
                        kj += 1
        self.data = np.zeros((len(self.col), block, block))
        self.lu = [None] * self.rows

    def at(self, i: int, j: int) -> int:
        lo, hi = self.row[i], self.row[i + 1]
        pos = lo + int(np.searchsorted(self.col[lo:hi], j))
        require(pos < hi and self.col[pos] == j, "Entry outside fixed BSR graph")
        return pos

    def factor(self):                                               # block_ilu.cpp:74-87
        import scipy.linalg as sla
        for i in range(self.rows):
            for ik in range(self.row[i], self.diag[i]):
                k = self.col[ik]
                # RightSolve: X <- X A_kk^{-1} with the pivoted LU of A_kk
                self.data[ik] = sla.lu_solve(self.lu[k], self.data[ik].T, trans=1).T
                for target, upper in self.updates[ik]:
                    self.data[target] -= self.data[ik] @ self.data[upper]
            a = self.data[self.diag[i]]
            lu, piv = sla.lu_factor(a, check_finite=False)
            require(np.all(np.isfinite(lu)) and np.all(np.diag(lu) != 0), "Singular BSR ILU diagonal")
            self.lu[i] = (lu, piv)

    def __call__(self, b):                                          # block_ilu.cpp:88-109
        import scipy.linalg as sla
        B = self.b
        w = np.array(b, float).reshape(self.rows, B)
        for i in range(self.rows):
            for ij in range(self.row[i], self.diag[i]):
                w[i] -= self.data[ij] @ w[self.col[ij]]
        for i in range(self.rows - 1, -1, -1):
            for ij in range(self.diag[i] + 1, self.row[i + 1]):
                w[i] -= self.data[ij] @ w[self.col[ij]]
            w[i] = sla.lu_solve(self.lu[i], w[i])
        return w.reshape(-1)


def fill_dg_ilu(pb: Problem, ilu: BlockILU0, u):
    """PartialDGOperator::FillBlocks (partial.cpp:140-170): cell blocks on the
    diagonal, face couplings l->r (+scale jr) and r->l (-scale jl) off it."""
    ilu.data[:] = 0.0
    diag = pb.dg_jacobi_blocks(u)                                    # also refreshes jl, jr
    for e in range(pb.n):
        ilu.data[ilu.at(e, e)] = diag[e]
    scale = (pb.dt * pb.face_len / pb.area)[:, None] * pb.tab.ew[None, :]
    tb = pb.tab
    for f in range(pb.nf):
        ls = 1 if f % 2 == 0 else 3
        rs = ls - 1
        l, r = int(pb.face_l[f]), int(pb.face_r[f])
        lr = np.einsum("j,ji,jl,jcd->icld", scale[f], tb.fv[ls] * tb.inv_mass[None, :], tb.fv[rs],
                       pb._jr[f]).reshape(pb.m, pb.m)
        rl = np.einsum("j,ji,jl,jcd->icld", -scale[f], tb.fv[rs] * tb.inv_mass[None, :], tb.fv[ls],
                       pb._jl[f]).reshape(pb.m, pb.m)
        ilu.data[ilu.at(l, r)] += lr
        ilu.data[ilu.at(r, l)] += rl


def fill_hdg_ilu(pb: Problem, ilu: BlockILU0):
    """ElementOperator::FillBlocks on the condensed operator (operators.cpp:48-74):
    D on the diagonal, minus every cell's panels C_s X_{s,o}."""
    t = pb.t
    ilu.data[:] = 0.0
    idx = np.arange(t)
    for f in range(pb.nf):
        ilu.data[ilu.at(f, f)][idx, idx] = pb.D[f * t:(f + 1) * t]
    panels = pb.schur_panels()
    for e in range(pb.n):
        for s in range(4):
            for o in range(4):
                ilu.data[ilu.at(int(pb.cell_faces[e, s]), int(pb.cell_faces[e, o]))] += -panels[e, s, o]


# ----------------------------------------------------------------------------
# Weighted CGS2 GMRES (src/linear.cpp:58-157, 167-249)
# ----------------------------------------------------------------------------

class BlockJacobi:
    """Block-Jacobi preconditioner: per-block pivoted LU solve (linear.cpp:66-75)."""

    def __init__(self, blocks: np.ndarray):
        self.blocks = blocks
        self.b = blocks.shape[1]
        if not np.all(np.isfinite(blocks)):
            raise OracleError("Singular block Jacobi factor")
        try:
            self.inv = np.linalg.inv(blocks)
        except np.linalg.LinAlgError as exc:
            raise OracleError("Singular block Jacobi factor") from exc

    def __call__(self, v):
        return np.linalg.solve(self.blocks, np.asarray(v, float).reshape(-1, self.b, 1)).reshape(-1)


def gmres(apply, precond, rhs, metric, tol: float, limit: int, restart: int, x0=None):
    """LinearSolver::Impl::GMRES (linear.cpp:76-157): right-preconditioned
    restarted GMRES with metric-weighted CGS2.  Returns (x, count,
    residual_norm, residual, rhs_norm)."""
    n = len(rhs)
    restart = min(n, restart)
    dot = lambda a, b: float(np.sum(metric * a * b))
    norm = lambda a: math.sqrt(dot(a, a))
    if x0 is None:
        x = np.zeros(n)
        residual = np.array(rhs, float)
    else:
        x = np.array(x0, float)
        residual = rhs - apply(x)
    rhs_norm = norm(rhs)
    if rhs_norm == 0.0:
        return x, 0, 0.0, residual, 0.0
    iterations = 0
    residual_norm = norm(residual)
    basis = np.zeros((restart + 1, n))
    while iterations < limit:
        beta = residual_norm
        if beta <= tol * rhs_norm:
            break
        basis[0] = residual * (1 / beta)
        h = np.zeros((restart + 1, restart))
        g = np.zeros(restart + 1)
        g[0] = beta
        cs, sn = np.zeros(restart), np.zeros(restart)
        count = 0
        for j in range(restart):
            if iterations >= limit:
                break
            w = apply(precond(basis[j]))
            for _ in range(2):                                   # CGS2, linear.cpp:109-121
                proj = basis[:j + 1] @ (metric * w)
                h[:j + 1, j] += proj
                w = w - basis[:j + 1].T @ proj
            nxt = norm(w)
            h[j + 1, j] = nxt
            if nxt > 0:
                basis[j + 1] = w * (1 / nxt)
            for i in range(j):
                u_, v_ = h[i, j], h[i + 1, j]
                h[i, j] = cs[i] * u_ + sn[i] * v_
                h[i + 1, j] = -sn[i] * u_ + cs[i] * v_
            d = math.hypot(h[j, j], h[j + 1, j])
            require(math.isfinite(d) and d > 0, "GMRES Arnoldi breakdown")
            cs[j], sn[j] = h[j, j] / d, h[j + 1, j] / d
            h[j, j], h[j + 1, j] = d, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] *= cs[j]
            iterations += 1
            count = j + 1
            if abs(g[j + 1]) <= tol * rhs_norm or nxt <= TINY:
                break
        coef = np.zeros(count)
        for i in range(count - 1, -1, -1):
            coef[i] = (g[i] - h[i, i + 1:count] @ coef[i + 1:count]) / h[i, i]
        x = x + precond(basis[:count].T @ coef)
        residual = rhs - apply(x)
        residual_norm = norm(residual)
        require(math.isfinite(residual_norm), "Nonfinite GMRES residual")
    require(residual_norm <= tol * rhs_norm, "GMRES iteration limit reached")
    return x, iterations, residual_norm, residual, rhs_norm


@dataclass
class LinearResult:
    x: np.ndarray
    equation_residual: np.ndarray
    count: int
    residual: float


def linear_solve(apply, precond_blocks, rhs, metric, linear_tol=1e-12, max_krylov=1500, restart=20,
                 x0=None, pc=None):
    """LinearSolver::Solve, matrix-free GMRES branch (linear.cpp:167-249).
    `precond_blocks` refreshes the block-Jacobi factors (refresh=true);
    passing `pc` and `x0` keeps old factors and warm-starts (refresh=false)."""
    n = len(rhs)
    pc = pc if pc is not None else None
    rn = math.sqrt(float(np.sum(metric * rhs * rhs)))
    if rn == 0.0:
        return LinearResult(np.zeros(n), np.zeros(n), 0, 0.0), pc
    if pc is None:
        pc = precond_blocks if callable(precond_blocks) else BlockJacobi(precond_blocks)
    x, count, res_norm, residual, rhs_norm = gmres(apply, pc, rhs, metric, linear_tol, max_krylov, restart, x0)
    rel = res_norm / rhs_norm
    require(math.isfinite(rel) and rel <= max(10 * linear_tol, 1e-12),
            "True inverse-mass weighted linear residual too large")
    return LinearResult(x, -residual, count, rel), pc


# ----------------------------------------------------------------------------
# Newton update and time loop (src/stepper.cpp:28-292)
# ----------------------------------------------------------------------------

SSP_ALPHA = 0.24169426078821
SSP_BETA = SSP_ALPHA / 4.0
SSP_ETA = 0.12915286960590
SSP_A = np.array([[SSP_ALPHA, 0, 0, 0], [-SSP_ALPHA, SSP_ALPHA, 0, 0], [0, 1 - SSP_ALPHA, SSP_ALPHA, 0],
                  [SSP_BETA, SSP_ETA, 0.5 - SSP_BETA - SSP_ETA - SSP_ALPHA, SSP_ALPHA]])
SSP_B = np.array([0.0, 1 / 6, 1 / 6, 2 / 3])
SSP_C = np.array([SSP_ALPHA, 0.0, 1.0, 0.5])


@dataclass
class UpdateRecord:
    rms: float
    damping: float
    krylov: int
    linear_relres: float
    dg_relres: float


def _preconditioner(pb: Problem, form: str, precond: str, u):
    """Refreshed preconditioner of the current form (linear.cpp:177-203)."""
    if precond == "block-ilu0":
        ilu = BlockILU0(solver_graph(pb, form == "hdg"), pb.t if form == "hdg" else pb.m)
        if form == "hdg":
            fill_hdg_ilu(pb, ilu)
        else:
            fill_dg_ilu(pb, ilu, u)
        ilu.factor()
        return ilu
    return BlockJacobi(pb.schur_jacobi_blocks() if form == "hdg" else pb.dg_jacobi_blocks(u))


def newton_update(pb: Problem, form: str, u, residual, old_norm: float, linear_tol=1e-12,
                  max_krylov=1500, restart=20, precond="block-jacobi"):
    """One accepted damped Newton update (stepper.cpp:136-224).  Returns the
    accepted state, its residual and the per-update record."""
    residual_norm = pb.cell_norm(residual)
    allowance = 128 * EPS * (pb.cell_norm(u) + old_norm + residual_norm)
    target = max(10 * linear_tol * residual_norm, allowance)
    if form == "dg":
        pb.dg_refresh(u)
        lr, _ = linear_solve(pb.dg_apply, _preconditioner(pb, form, precond, u), -residual, pb.cell_metric,
                             linear_tol, max_krylov, restart)
        du = lr.x
        er_norm = pb.cell_norm(lr.equation_residual)
        count, lrel = lr.count, lr.residual
    else:
        _, _, rhs, _ = pb.condense(u, residual)
        blocks = _preconditioner(pb, form, precond, u)
        tol = linear_tol
        valid = False
        count = 0
        pc = None
        x = None
        for attempt in range(4):                                  # stepper.cpp:159-179
            lr, pc = linear_solve(pb.schur_apply, blocks, rhs, pb.trace_metric, tol, max_krylov, restart,
                                  x0=None if attempt == 0 else x, pc=None if attempt == 0 else pc)
            x = lr.x
            count += lr.count
            lrel = lr.residual
            du = pb.recover(lr.x)
            er_norm = pb.cell_norm(pb.recovered_residual(lr.equation_residual))
            valid = er_norm <= target
            if valid:
                break
            tol *= 0.01
        require(valid, "Recovered DG residual criterion failed after Schur refinement")
    dgrel = er_norm / residual_norm if residual_norm > 0 else 0.0
    require(er_norm <= target, "DG Newton linear residual too large")
    damping = 1.0
    for _ in range(30):                                           # stepper.cpp:203-216
        trial = u + damping * du
        if pb.admissible(trial):
            tr = pb.residual(trial)
            if pb.cell_norm(tr) <= (1 - 1e-4 * damping) * residual_norm + allowance:
                return trial, tr, (damping, count, lrel, dgrel)
        damping *= 0.5
    raise OracleError("Newton line search failed")


def run(nx, ny, k, alpha_deg, form="hdg", cfl=1.0, steps=1, newton_steps=1, integrator="ssp-dirk3",
        linear_tol=1e-12, max_krylov=1500, restart=20, safety=1.1, gamma=3.0, u0=None, tables=None,
        precond="block-jacobi"):
    """Run() for a fixed number of steps and Newton updates per stage
    (stepper.cpp:28-292, the `--steps N --newton-steps M --cfl C` branch).
    Returns (u, records) with one UpdateRecord per update."""
    pb = Problem(nx, ny, k, alpha_deg, safety, gamma, tables)
    u = pb.initial() if u0 is None else np.array(u0, float)
    require(pb.admissible(u), "Initial projection not positive; refine mesh")
    records = []
    time = 0.0
    slopes = [None] * 4
    for _step in range(steps):
        step_state = u.copy()
        rate = pb.freeze(step_state, 0.001, False)
        dt = cfl / rate
        require(math.isfinite(dt) and dt > 0 and time + dt < 4 / ((gamma + 1) * PI),
                "Step leaves the smooth simple-wave interval T < 4/((gamma+1)*pi)")
        nst = 1 if integrator == "be" else 4
        for stage in range(nst):
            diag = 1.0 if integrator == "be" else SSP_A[stage, stage]
            base = step_state.copy()
            if integrator != "be":
                for j in range(stage):
                    base = base + dt * SSP_A[stage, j] * slopes[j]
            if stage > 0:
                pb.freeze(u, diag * dt, False)
            pb.dt = diag * dt
            pb.old = base
            phys = 1 / (pb.dt * math.sqrt(pb.lx * pb.ly))
            old_norm = pb.cell_norm(base)
            residual = None
            for _it in range(newton_steps):
                if residual is None:
                    residual = pb.residual(u)
                rms = phys * pb.cell_norm(residual)
                u, residual, (damping, count, lrel, dgrel) = newton_update(
                    pb, form, u, residual, old_norm, linear_tol, max_krylov, restart, precond)
                records.append(UpdateRecord(rms, damping, count, lrel, dgrel))
            slopes[stage] = (u - base) * (1.0 / pb.dt)
        if integrator != "be":
            u = step_state.copy()
            for stage in range(4):
                u = u + dt * SSP_B[stage] * slopes[stage]
            require(pb.admissible(u), "SSP-DIRK3 step produced an inadmissible state")
        time += dt
    return u, records, pb, time
