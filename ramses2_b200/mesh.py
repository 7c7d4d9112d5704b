"""Flat-oct meshes in the reference layout, and the synthetic initial conditions.

A :class:`Mesh` holds exactly what RAMSES II's ``mesh_t`` holds for the hydro
step (amr/amr_commons.f90:811-920): ``grid(1:N)`` oct records, ``uold(1:8,
1:nvar,1:N)`` (numpy shape ``(N, 5, 8)``, C order, so oct ``igrid`` is the
40-double record at ``uold[igrid-1]``), and per-level ``head``/``noct``.
Octs of a level are contiguous and grouped in blocks of ``nsubgrid**3``
consecutive octs forming an aligned cube, as ``godunov_fine`` expects
(hydro/godunov_fine.f90:72-74).  Cell ``ind`` (0-based) of an oct has offsets
``(ind&1, ind>>1&1, ind>>2&1)``; its centre is ``(2*ckey+offset+0.5)*dx``
(hydro/courant_fine.f90:200-204).
"""
import ctypes as C

import numpy as np

from ._abi import OCT_DTYPE, MeshDesc, RH_BOUND_PERIODIC, RH_BOUND_REFLEXIVE, RH_BOUND_ZERO_GRADIENT

BC_NAMES = {"periodic": RH_BOUND_PERIODIC, "reflexive": RH_BOUND_REFLEXIVE,
            "outflow": RH_BOUND_ZERO_GRADIENT, "zero_gradient": RH_BOUND_ZERO_GRADIENT}

CELL_OFF = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.int64)


def _morton3(x, y, z, bits=21):
    """Interleave the bits of three non-negative int arrays (x fastest)."""
    key = np.zeros(np.broadcast(x, y, z).shape, dtype=np.int64)
    x = np.asarray(x, np.int64)
    y = np.asarray(y, np.int64)
    z = np.asarray(z, np.int64)
    for b in range(bits):
        key |= ((x >> b) & 1) << (3 * b)
        key |= ((y >> b) & 1) << (3 * b + 1)
        key |= ((z >> b) & 1) << (3 * b + 2)
    return key


class Mesh:
    """Reference-layout mesh: grid records, uold, level ranges, box and BCs."""

    def __init__(self, grid, levelmin, levelmax, nsubgrid=1, boxlen=1.0, bc="outflow",
                 box_nx=(1, 1, 1), gravity=(0.0, 0.0, 0.0), ngridmax=None):
        self.grid = np.ascontiguousarray(grid, dtype=OCT_DTYPE)
        n = len(self.grid)
        self.levelmin = int(levelmin)
        self.levelmax = int(levelmax)
        self.nsubgrid = int(nsubgrid)
        self.boxlen = float(boxlen)
        self.box_nx = tuple(int(v) for v in box_nx)
        self.gravity = tuple(float(v) for v in gravity)
        self.ngridmax = int(ngridmax if ngridmax is not None else n)
        if isinstance(bc, str):
            bc = [BC_NAMES[bc]] * 6
        self.bound_type = [int(BC_NAMES[b]) if isinstance(b, str) else int(b) for b in bc]
        assert len(self.bound_type) == 6
        self.periodic = [int(self.bound_type[2 * d] == RH_BOUND_PERIODIC) for d in range(3)]
        self.head = np.zeros(self.levelmax + 1, dtype=np.int32)
        self.noct = np.zeros(self.levelmax + 1, dtype=np.int32)
        levs = self.grid["lev"]
        for lev in range(1, self.levelmax + 1):
            idx = np.nonzero(levs == lev)[0]
            if len(idx):
                assert np.all(np.diff(idx) == 1), "octs of a level must be contiguous"
                self.head[lev] = idx[0] + 1
                self.noct[lev] = len(idx)
        self.uold = np.zeros((self.ngridmax, 5, 8), dtype=np.float64)
        self._desc = None

    # -- geometry ---------------------------------------------------------
    @property
    def noct_total(self):
        return len(self.grid)

    def dx(self, lev):
        return self.boxlen / 2.0 ** lev

    def level_slice(self, lev):
        h = int(self.head[lev])
        return slice(h - 1, h - 1 + int(self.noct[lev]))

    def cell_centres(self, lev):
        """(noct, 8, 3) cell-centre coordinates of level ``lev``."""
        g = self.grid[self.level_slice(lev)]
        ck = g["ckey"].astype(np.int64)
        return ((2 * ck[:, None, :] + CELL_OFF[None, :, :]) + 0.5) * self.dx(lev)

    def leaf_mask(self, lev):
        return self.grid[self.level_slice(lev)]["refined"] == 0

    def ncells_leaf(self):
        return int(sum(self.leaf_mask(l).sum() for l in range(self.levelmin, self.levelmax + 1)
                       if self.noct[l]))

    # -- C view -----------------------------------------------------------
    def desc(self):
        """rh_mesh_desc pointing at this mesh's arrays (kept alive by self)."""
        d = MeshDesc()
        d.nsubgrid = self.nsubgrid
        d.levelmin = self.levelmin
        d.levelmax = self.levelmax
        d.ngridmax = self.ngridmax
        for i in range(3):
            d.box_nx[i] = self.box_nx[i]
            d.periodic[i] = self.periodic[i]
            d.constant_gravity[i] = self.gravity[i]
        for i in range(6):
            d.bound_type[i] = self.bound_type[i]
        d.boxlen = self.boxlen
        d.head = self.head.ctypes.data_as(C.POINTER(C.c_int32))
        d.noct = self.noct.ctypes.data_as(C.POINTER(C.c_int32))
        d.grid = self.grid.ctypes.data
        self._desc = d
        return d

    # -- dense views (uniform levels) ------------------------------------
    def to_dense(self, u, lev):
        """Scatter a level of a (N,5,8) state into a dense (5,nz,ny,nx) array."""
        g = self.grid[self.level_slice(lev)]
        ck = g["ckey"].astype(np.int64)
        n = [self.box_nx[d] << lev for d in range(3)]
        out = np.zeros((5, n[2], n[1], n[0]), dtype=u.dtype)
        cells = 2 * ck[:, None, :] + CELL_OFF[None, :, :]
        ux = u[self.level_slice(lev)]  # (noct,5,8)
        for v in range(5):
            out[v, cells[..., 2], cells[..., 1], cells[..., 0]] = ux[:, v, :]
        return out

    def from_dense(self, dense, lev):
        g = self.grid[self.level_slice(lev)]
        ck = g["ckey"].astype(np.int64)
        cells = 2 * ck[:, None, :] + CELL_OFF[None, :, :]
        sl = self.level_slice(lev)
        for v in range(5):
            self.uold[sl, v, :] = dense[v, cells[..., 2], cells[..., 1], cells[..., 0]]


def _demorton3(key, bits=21):
    """Inverse of :func:`_morton3`: (x, y, z) of interleaved keys."""
    key = np.asarray(key, np.int64)
    out = []
    for d in range(3):
        v = np.zeros(key.shape, dtype=np.int64)
        for b in range(bits):
            v |= ((key >> (3 * b + d)) & 1) << b
        out.append(v)
    return out


def uniform_mesh(level, nsubgrid=1, boxlen=1.0, bc="outflow", gravity=(0.0, 0.0, 0.0), box_nx=(1, 1, 1)):
    """A single-level mesh (levelmin = levelmax = level) covering its box.

    ``box_nx`` is the box size in level-1 octs (a level-l edge holds
    ``box_nx[d] * 2**(l-1)`` octs).  Blocks of nsubgrid**3 octs are stored in
    Morton order of the block coordinate, octs inside a block in Morton order.
    """
    no = [int(box_nx[d]) << (level - 1) for d in range(3)]
    assert all(n % nsubgrid == 0 for n in no), "octs per edge must be a multiple of nsubgrid"
    if nsubgrid == 1 and tuple(box_nx) == (1, 1, 1):
        # a 2^k cube: the Morton keys of its octs are exactly 0 .. N-1
        key = np.arange(no[0] ** 3, dtype=np.int64)
        x, y, z = _demorton3(key, bits=level)
        grid = np.zeros(len(key), dtype=OCT_DTYPE)
        grid["ckey"][:, 0] = x
        grid["ckey"][:, 1] = y
        grid["ckey"][:, 2] = z
        grid["lev"] = level
        grid["hkey"] = key
        return Mesh(grid, level, level, nsubgrid=1, boxlen=boxlen, bc=bc, gravity=gravity, box_nx=box_nx)
    ix, iy, iz = np.meshgrid(np.arange(no[0]), np.arange(no[1]), np.arange(no[2]), indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    n = nsubgrid
    bkey = _morton3(ix // n, iy // n, iz // n)
    okey = _morton3(ix % n, iy % n, iz % n)
    order = np.lexsort((okey, bkey))
    grid = np.zeros(len(ix), dtype=OCT_DTYPE)
    grid["ckey"][:, 0] = ix[order]
    grid["ckey"][:, 1] = iy[order]
    grid["ckey"][:, 2] = iz[order]
    grid["lev"] = level
    grid["hkey"] = _morton3(ix[order], iy[order], iz[order])
    return Mesh(grid, level, level, nsubgrid=nsubgrid, boxlen=boxlen, bc=bc, gravity=gravity, box_nx=box_nx)


# ---------------------------------------------------------------------------
# Conserved <-> primitive (hydro/courant_fine.f90:219-235 reset_init form)
# ---------------------------------------------------------------------------
def prim_to_cons(rho, u, v, w, p, gamma):
    ekin = 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
    eint = p / (gamma - 1.0)
    return np.stack([rho, rho * u, rho * v, rho * w, eint + ekin])


def set_level_prim(mesh, lev, rho, u, v, w, p, gamma):
    """Fill uold of a level from per-cell primitive arrays of shape (noct, 8)."""
    cons = prim_to_cons(rho, u, v, w, p, gamma)  # (5, noct, 8)
    mesh.uold[mesh.level_slice(lev)] = np.transpose(cons, (1, 0, 2))


# ---------------------------------------------------------------------------
# Initial conditions
# ---------------------------------------------------------------------------
def sedov3d(mesh, gamma=1.4, rho0=1.0, p0=1e-5, energy=1.0, radius_cells=2.0, centre=None):
    """Sedov blast: ambient (rho0, v=0, p0); total energy ``energy`` spread as a
    uniform pressure over the finest-level cells whose centres lie within
    ``radius_cells`` cells of the box centre (every level gets the same
    pressure inside the sphere so the coarse cells agree)."""
    lmax = max(l for l in range(mesh.levelmin, mesh.levelmax + 1) if mesh.noct[l])
    dxf = mesh.dx(lmax)
    c = np.array(centre if centre is not None else
                 [0.5 * mesh.boxlen * mesh.box_nx[d] for d in range(3)])
    rad = radius_cells * dxf * (1 + 1e-12)

    def near(lev):
        """Octs of a level whose cells can lie within the radius, and the
        centre distances of their cells (same arithmetic as cell_centres)."""
        ck = mesh.grid[mesh.level_slice(lev)]["ckey"].astype(np.int64)
        dx = mesh.dx(lev)
        oc = (2 * ck + 1) * dx
        cand = np.nonzero(np.sqrt(((oc - c) ** 2).sum(-1)) <= rad + 2 * dx)[0]
        x = ((2 * ck[cand][:, None, :] + CELL_OFF[None, :, :]) + 0.5) * dx
        return cand, np.sqrt(((x - c) ** 2).sum(-1))

    cand, rf = near(lmax)
    n_in = int((rf <= rad).sum())
    assert n_in > 0
    p_in = (gamma - 1.0) * energy / (n_in * dxf ** 3)
    amb = prim_to_cons(np.float64(rho0), 0.0, 0.0, 0.0, np.float64(p0), gamma)
    blast = prim_to_cons(np.float64(rho0), 0.0, 0.0, 0.0, np.float64(p_in), gamma)
    for lev in range(mesh.levelmin, mesh.levelmax + 1):
        if not mesh.noct[lev]:
            continue
        sl = mesh.level_slice(lev)
        mesh.uold[sl] = amb[None, :, None]
        cand, r = near(lev)
        o, cell = np.nonzero(r <= rad)
        for v in range(5):
            mesh.uold[sl.start + cand[o], v, cell] = blast[v]
    return n_in, p_in


def turbulence3d(mesh, gamma=1.001, mach=5.0, sigma_lnrho=0.1, kmin=1, kmax=4, seed=20261203):
    """Decaying supersonic turbulence (uniform mesh): Gaussian random-phase
    solenoidal velocity with P(k) ~ k^-2 on kmin<=|k|<=kmax (the recipe of
    utils/py/grafic/turb.py, alpha=0 projection), rms Mach ``mach`` for a unit
    mean sound speed, lognormal density of log-sigma ``sigma_lnrho``."""
    lev = mesh.levelmin
    n = [mesh.box_nx[d] << lev for d in range(3)]
    assert n[0] == n[1] == n[2]
    N = n[0]
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(N, d=1.0 / N)
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    band = (kk >= kmin) & (kk <= kmax)
    filt = np.zeros_like(kk)
    filt[band] = np.sqrt(kk[band] ** -2.0)  # power per mode ~ k^-2
    vel = [np.fft.fftn(rng.standard_normal(kk.shape)) * filt for _ in range(3)]
    # solenoidal projection: v_k - k (k.v_k)/k^2
    kk2 = np.where(kk > 0, kk ** 2, 1.0)
    dot = (kx * vel[0] + ky * vel[1] + kz * vel[2]) / kk2
    vel = [vel[0] - kx * dot, vel[1] - ky * dot, vel[2] - kz * dot]
    v = [np.real(np.fft.ifftn(c)) for c in vel]
    vrms = np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    cs = 1.0
    v = [c * (mach * cs / vrms) for c in v]
    g = rng.standard_normal((N, N, N))
    gk = np.fft.fftn(g)
    gk[~band & (kk > 0)] *= 0.0
    g = np.real(np.fft.ifftn(gk))
    g /= max(g.std(), 1e-300)
    rho = np.exp(sigma_lnrho * g - 0.5 * sigma_lnrho ** 2)
    p = np.full_like(rho, cs ** 2 * np.mean(rho) / gamma)
    # dense arrays are indexed [x,y,z]; Mesh.from_dense wants (5, z, y, x)
    dense = prim_to_cons(rho, v[0], v[1], v[2], p, gamma)
    dense = np.ascontiguousarray(np.transpose(dense, (0, 3, 2, 1)))
    mesh.from_dense(dense, lev)
    return mesh


def riemann3d_state(rng, n_cells, gamma=None):
    """One random 3D Riemann/blast problem as in the batched ensemble:
    states split along a random axis, rho log-uniform in [1e-3,1e3], p
    log-uniform in [1e-4,1e2], |v| uniform in [0,3] c_s, gamma in [1.1,1.67].
    Returns (gamma, dense conserved (5, n, n, n) indexed [v, z, y, x])."""
    g = float(gamma if gamma is not None else rng.uniform(1.1, 1.67))
    axis = int(rng.integers(0, 3))
    N = n_cells
    states = []
    for _ in range(2):
        rho = 10 ** rng.uniform(-3, 3)
        p = 10 ** rng.uniform(-4, 2)
        cs = np.sqrt(g * p / rho)
        vmag = rng.uniform(0, 3) * cs
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        states.append((rho, *(vmag * d), p))
    idx = np.arange(N)
    left = (idx < N // 2)
    shape = [1, 1, 1]
    shape[2 - axis] = N  # dense is [z, y, x]
    mask = left.reshape(shape)
    mask = np.broadcast_to(mask, (N, N, N))
    prims = [np.where(mask, states[0][i], states[1][i]) for i in range(5)]
    return g, prim_to_cons(*prims, g)


# ---------------------------------------------------------------------------
# Static AMR meshes
# ---------------------------------------------------------------------------
def _shift_reduce(a, r, op, fill):
    """Separable Chebyshev-window reduction (op = np.logical_or / logical_and)
    of a dense boolean grid over offsets -r..r per axis; outside the grid
    counts as ``fill``."""
    out = a
    for ax in range(a.ndim):
        pad = [(0, 0)] * a.ndim
        pad[ax] = (r, r)
        p = np.pad(out, pad, constant_values=fill)
        acc = None
        n = out.shape[ax]
        for k in range(2 * r + 1):
            sl = [slice(None)] * a.ndim
            sl[ax] = slice(k, k + n)
            v = p[tuple(sl)]
            acc = v.copy() if acc is None else op(acc, v, out=acc)
        out = acc
    return out


def amr_mesh(levelmin, levelmax, refine, bc="outflow", boxlen=1.0, nexpand=1, box_nx=(1, 1, 1)):
    """Properly nested static AMR mesh (nsubgrid = 1).

    Level ``levelmin`` fills the box.  At each level l < levelmax, the cells
    for which ``refine(centres (n,3), l)`` is true, dilated by ``nexpand`` cells
    and restricted to cells at least 2 cells (in every direction) inside the
    level's covered region, get a child oct at level l+1 - the margin that
    interpolating a missing fine neighbour needs (father cell and its six
    neighbours, hydro/interpol_hydro.f90:5-109).  Out-of-box neighbours do not
    count against the margin.  Octs are stored level by level in Morton order,
    and ``refined`` flags mark the cells that have children.  Works on dense
    boolean grids of each level's cells (one byte per cell of the level's box).
    """
    nb = np.array(box_nx, dtype=np.int64)
    levels = {}
    no = nb << (levelmin - 1)
    ix, iy, iz = np.meshgrid(np.arange(no[0]), np.arange(no[1]), np.arange(no[2]), indexing="ij")
    levels[levelmin] = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.int64)
    for l in range(levelmin, levelmax):
        octs = levels[l]
        cells = (2 * octs[:, None, :] + CELL_OFF[None, :, :]).reshape(-1, 3)
        dx = boxlen / 2.0 ** l
        flag = np.asarray(refine((cells + 0.5) * dx, l), dtype=bool)
        if not flag.any():
            break
        ncell = tuple(int(v) for v in (nb << l))
        F = np.zeros(ncell, dtype=bool)
        fc = cells[flag]
        F[fc[:, 0], fc[:, 1], fc[:, 2]] = True
        if nexpand > 0:
            F = _shift_reduce(F, nexpand, np.logical_or, False)
        cov = np.zeros(ncell, dtype=bool)
        cov[cells[:, 0], cells[:, 1], cells[:, 2]] = True
        # margin: every in-box cell within 2 of a candidate must exist at level l
        F &= _shift_reduce(cov, 2, np.logical_and, True)
        fk = np.argwhere(F).astype(np.int64)
        if len(fk) == 0:
            break
        levels[l + 1] = fk  # child oct keys at level l+1 = flagged cell coords (lexicographic)
    lmax = max(levels)
    grids = []
    for l in range(levelmin, lmax + 1):
        k = levels[l]
        order = np.argsort(_morton3(k[:, 0], k[:, 1], k[:, 2]), kind="stable")
        k = k[order]
        levels[l] = k
        g = np.zeros(len(k), dtype=OCT_DTYPE)
        g["ckey"] = k
        g["lev"] = l
        g["hkey"] = _morton3(k[:, 0], k[:, 1], k[:, 2])
        if l < lmax:
            ncell = tuple(int(v) for v in (nb << l))
            ch = np.zeros(ncell, dtype=bool)
            kc = levels[l + 1]
            ch[kc[:, 0], kc[:, 1], kc[:, 2]] = True
            cells = 2 * k[:, None, :] + CELL_OFF[None, :, :]
            g["refined"] = ch[cells[..., 0], cells[..., 1], cells[..., 2]].astype(np.uint8)
        grids.append(g)
    grid = np.concatenate(grids)
    return Mesh(grid, levelmin, lmax, nsubgrid=1, boxlen=boxlen, bc=bc, box_nx=box_nx)


def fill_amr_prim(mesh, prim_fn, gamma):
    """Fill every level from a function of cell centres -> (rho, u, v, w, p)."""
    for lev in range(mesh.levelmin, mesh.levelmax + 1):
        if not mesh.noct[lev]:
            continue
        x = mesh.cell_centres(lev)
        rho, u, v, w, p = prim_fn(x, lev)
        set_level_prim(mesh, lev, rho, u, v, w, p, gamma)


# ---------------------------------------------------------------------------
# Gradient refinement criterion and a developed Sedov-like blast (the AMR Sedov mesh)
# ---------------------------------------------------------------------------
def hydro_refine_flags(prim_fn, x, dx, err_grad_d=0.1, err_grad_p=0.1, floor_d=1e-10, floor_p=1e-10):
    """hydro_refine's density and pressure criteria (hydro/godunov_utils.f90:
    6-223): a cell is flagged when, along some axis, 2 max(|d_r - d|/(d_r + d
    + floor), |d - d_l|/(d + d_l + floor)) exceeds err_grad (same for p), with
    the left/right neighbours at x -+ dx.  ``prim_fn(x) -> (rho, u, v, w, p)``."""
    rho, _, _, _, p = prim_fn(x)
    ok = np.zeros(x.shape[:-1], dtype=bool)
    for d in range(3):
        e = np.zeros(3)
        e[d] = dx
        rl, _, _, _, pl = prim_fn(x - e)
        rr, _, _, _, pr = prim_fn(x + e)
        ed = 2.0 * np.maximum(np.abs((rr - rho) / (rr + rho + floor_d)), np.abs((rho - rl) / (rho + rl + floor_d)))
        ep = 2.0 * np.maximum(np.abs((pr - p) / (pr + p + floor_p)), np.abs((p - pl) / (p + pl + floor_p)))
        ok |= (ed > err_grad_d) | (ep > err_grad_p)
    return ok


def sedov_like_blast(radius=0.2, gamma=1.4, energy=1.0, rho0=1.0, p0=1e-5, centre=(0.5, 0.5, 0.5), rho_floor=1e-3):
    """Primitive state of a developed point blast with its shock at ``radius``:
    strong-shock jump conditions at the front, a steep density profile
    rho ~ (r/R)^(3/(gamma-1)) behind it, velocity linear in r and a pressure
    plateau at 30 % of the post-shock value (a closed-form stand-in for the
    self-similar Sedov-Taylor profile).  Returns prim_fn(x) -> (rho, u, v, w, p)."""
    xi = 1.15  # Sedov constant for gamma = 1.4 in 3D
    t = np.sqrt(radius ** 5 * rho0 / (xi ** 5 * energy))
    rdot = 0.4 * radius / t
    rho1 = rho0 * (gamma + 1) / (gamma - 1)
    v1 = 2.0 / (gamma + 1) * rdot
    p1 = 2.0 / (gamma + 1) * rho0 * rdot ** 2
    c = np.asarray(centre, dtype=np.float64)

    def prim(x):
        dxv = x - c
        r = np.sqrt((dxv ** 2).sum(-1))
        s = np.minimum(r / radius, 1.0)
        inside = r < radius
        rho = np.where(inside, np.maximum(rho1 * s ** (3.0 / (gamma - 1)), rho_floor), rho0)
        vr = np.where(inside, v1 * s, 0.0)
        p = np.where(inside, p1 * (0.3 + 0.7 * s ** 8), p0)
        with np.errstate(invalid="ignore", divide="ignore"):
            nvec = np.where(r[..., None] > 0, dxv / np.maximum(r, 1e-300)[..., None], 0.0)
        return rho, vr * nvec[..., 0], vr * nvec[..., 1], vr * nvec[..., 2], p

    return prim


def sedov_amr_mesh(levelmin=7, levelmax=10, radius=0.2, gamma=1.4, err_grad=0.1, bc="outflow"):
    """AMR Sedov mesh: levels levelmin..levelmax refined where
    hydro_refine's relative density/pressure gradient exceeds ``err_grad`` on
    a developed Sedov-like blast (:func:`sedov_like_blast`), filled with that
    state.  Returns (mesh, gamma)."""
    prim = sedov_like_blast(radius=radius, gamma=gamma)
    m = amr_mesh(levelmin, levelmax,
                 lambda x, l: hydro_refine_flags(prim, x, 1.0 / 2 ** l, err_grad, err_grad), bc=bc)
    fill_amr_prim(m, lambda x, l: prim(x), gamma)
    return m, gamma

