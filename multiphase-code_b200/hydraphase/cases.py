"""Synthetic cases in the reference's input formats.

Meshes are hexahedral grids split into 6 tetrahedra per hex (Kuhn /
Freudenthal split along the main diagonal, conforming across hexes), with
every tet positively oriented (det[p2-p1, p3-p1, p4-p1] > 0) as the
reference's face-vector formula expects (src/sr_geometry.F90:147-189: face k
is opposite node k and its area vector points outward).  Cells are randomly
permuted (seeded) so that the engine's own renumbering is exercised.

Initial states are injected the way the reference accepts non-uniform ones:
as a restart (cu for the elements plus ug,vg,wg,pg,tg,rog at the ghosts,
src/main.F90:427-441).

Boundary types: 2 inflow, 3 outflow, 5 slip wall, 51/53 lateral (as in the
reference), plus 6 (no-slip isothermal wall) and 7 (far field) of this build.
"""
from __future__ import annotations

import itertools
import os
from dataclasses import dataclass

import numpy as np

from .engine import MeshArrays, make_params

R_GAS = 287.0
_PERMS = list(itertools.permutations(range(3)))


# ---------------------------------------------------------------------------
def _kuhn_tets(base: np.ndarray, corner) -> np.ndarray:
    """6 tets per hex; corner(dx,dy,dz) gives node ids of the hex corners."""
    tets = []
    for p in _PERMS:
        v = [0, 0, 0]
        ids = [corner(0, 0, 0)]
        for ax in p:
            v[ax] = 1
            ids.append(corner(*v))
        tets.append(np.stack(ids, axis=1))
    return np.stack(tets, axis=1).reshape(-1, 4)


def _orient(nod: np.ndarray, xyz: np.ndarray) -> np.ndarray:
    p = xyz[nod]
    d = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
    nod = nod.copy()
    neg = d < 0
    nod[neg, 2], nod[neg, 3] = nod[neg, 3].copy(), nod[neg, 2].copy()
    return nod


def _connect(nod: np.ndarray):
    """Face neighbours (0-based, -1 on the boundary) of tets; face k opposite node k."""
    ne = nod.shape[0]
    faces = np.stack([np.delete(nod, k, axis=1) for k in range(4)], axis=1)  # (ne,4,3)
    f = np.sort(faces.reshape(-1, 3).astype(np.int64), axis=1)
    key = (f[:, 0] << 42) | (f[:, 1] << 21) | f[:, 2]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    nb = np.full(4 * ne, -1, np.int64)
    same = np.where(ks[1:] == ks[:-1])[0]
    a, b = order[same], order[same + 1]
    nb[a] = b // 4
    nb[b] = a // 4
    return nb.reshape(ne, 4)


@dataclass
class Built:
    mesh: MeshArrays
    xc: np.ndarray        # element centroids (reference order), (neles, 3)
    vol: np.ndarray


def _assemble(xyz, nod, bc_type_fn, seed):
    """Permute cells, number ghosts, fill the reference's arrays."""
    nod = _orient(nod, xyz)
    ne = nod.shape[0]
    nb = _connect(nod)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(ne)            # new position of old tet
    inv = np.empty(ne, np.int64)
    inv[perm] = np.arange(ne)
    nod = nod[inv]
    nb = nb[inv]
    nb = np.where(nb >= 0, perm[np.maximum(nb, 0)], -1)
    # boundary faces -> ghosts, in (cell, face) order
    bcell, bface = np.nonzero(nb < 0)
    fn = np.array([np.delete(np.arange(4), k) for k in range(4)])
    fnodes = nod[bcell[:, None], fn[bface]]          # (nb,3)
    fcen = xyz[fnodes].mean(axis=1)
    btype = bc_type_fn(fcen).astype(np.int32)
    ng = bcell.size
    gid = ne + 1 + np.arange(ng)
    nc = nb + 1
    nc[bcell, bface] = gid
    elem = np.zeros((ne, 9), np.int32)
    elem[:, 0:4] = nod + 1
    elem[:, 4:8] = nc
    elem[:, 8] = 1
    ghost = np.stack([bcell + 1, gid, btype, bface + 1], axis=1).astype(np.int32)
    mesh = MeshArrays(xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy(), elem, ghost)
    p = xyz[nod]
    xc = p.mean(axis=1)
    vol = np.abs(np.einsum("ij,ij->i", p[:, 1] - p[:, 0],
                           np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))) / 6.0
    return Built(mesh, xc, vol)


def box_mesh(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=0,
             bc_type=5) -> Built:
    """Box of nx*ny*nz hexes split into 6 tets; interior nodes jittered by
    U(-jitter*h, +jitter*h) per axis; all boundary faces of type bc_type
    (an int or a function of the face centroids)."""
    rng = np.random.default_rng(seed)
    xs = [np.linspace(lo[d], hi[d], n + 1) for d, n in enumerate((nx, ny, nz))]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    xyz = np.stack([X, Y, Z], axis=-1).reshape(-1, 3).copy()
    if jitter > 0:
        h = np.array([(hi[d] - lo[d]) / n for d, n in enumerate((nx, ny, nz))])
        idx = np.stack(np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                                   indexing="ij"), axis=-1).reshape(-1, 3)
        interior = np.all((idx > 0) & (idx < np.array([nx, ny, nz])), axis=1)
        d = rng.uniform(-jitter, jitter, size=(interior.sum(), 3)) * h
        xyz[interior] += d

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    nod = _kuhn_tets(None, lambda a, b, c: nid(I + a, J + b, K + c))
    fn = bc_type if callable(bc_type) else (lambda fc: np.full(fc.shape[0], bc_type))
    return _assemble(xyz, nod, fn, seed)


def ogrid_mesh(nr, nt, nz, r_in=0.5, r_out=20.0, dr0=0.005, span=4.0, seed=1,
               wall_type=6, far_type=7, side_type=53) -> Built:
    """O-grid around a cylinder of diameter 2*r_in: nr radial cells with
    geometric stretching from dr0 at the wall to r_out, nt azimuthal cells
    (periodic), nz spanwise cells over `span`."""
    # geometric ratio q: dr0 * (q^nr - 1) / (q - 1) = r_out - r_in
    L = r_out - r_in
    lo_q, hi_q = 1.0 + 1e-12, 2.0
    for _ in range(200):
        q = 0.5 * (lo_q + hi_q)
        if dr0 * (q ** nr - 1) / (q - 1) > L:
            hi_q = q
        else:
            lo_q = q
    r = r_in + dr0 * (q ** np.arange(nr + 1) - 1) / (q - 1)
    r[-1] = r_out
    th = 2 * np.pi * np.arange(nt) / nt
    zz = np.linspace(0.0, span, nz + 1)
    Rr, Tt, Zz = np.meshgrid(r, th, zz, indexing="ij")
    xyz = np.stack([Rr * np.cos(Tt), Rr * np.sin(Tt), Zz], axis=-1).reshape(-1, 3).copy()

    def nid(i, j, k):
        return (i * nt + (j % nt)) * (nz + 1) + k

    I, J, K = np.meshgrid(np.arange(nr), np.arange(nt), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    nod = _kuhn_tets(None, lambda a, b, c: nid(I + a, J + b, K + c))

    def types(fc):
        rad = np.hypot(fc[:, 0], fc[:, 1])
        t = np.full(fc.shape[0], side_type)
        t[rad < 0.5 * (r[0] + r[1])] = wall_type
        t[rad > 0.5 * (r[-1] + r[-2])] = far_type
        return t

    return _assemble(xyz, nod, types, seed)


# ---------------------------------------------------------------------------
# conserved state from primitives (pressure equilibrium, sigma = 0)
def conserved(alpha_g, p, rho_g, rho_p, u, gamag, gamap, pinf):
    """cu (10, n) for phase fractions alpha_g, common pressure p, phase
    densities and a common velocity u (n, 3)."""
    ag = np.asarray(alpha_g, float)
    ap = 1.0 - ag
    ke = 0.5 * np.sum(u * u, axis=1)
    eg = p / ((gamag - 1.0) * rho_g)
    ep = (p + gamap * pinf) / ((gamap - 1.0) * rho_p)
    cu = np.empty((10, ag.size))
    cu[0] = ag * rho_g
    cu[1:4] = (ag * rho_g)[None] * u.T
    cu[4] = ag * rho_g * (eg + ke)
    cu[5] = ap * rho_p
    cu[6:9] = (ap * rho_p)[None] * u.T
    cu[9] = ap * rho_p * (ep + ke)
    return cu


def ghost_prims_from_parents(mesh: MeshArrays, cu, gamag, gamap, pinf):
    """ug,vg,wg,pg,tg,rog at the ghosts, copied from their parents."""
    par = mesh.ghost[:, 0] - 1
    c = cu[:, par]
    ug, vg, wg = c[1] / c[0], c[2] / c[0], c[3] / c[0]
    # air pressure from the equilibrium recovery with sigma = 0
    up, vp, wp = c[6] / c[5], c[7] / c[5], c[8] / c[5]
    eg = c[4] / c[0] - 0.5 * (ug ** 2 + vg ** 2 + wg ** 2)
    ep = c[9] / c[5] - 0.5 * (up ** 2 + vp ** 2 + wp ** 2)
    bbb = pinf * gamap - c[0] * (gamag - 1) * eg - c[5] * (gamap - 1) * ep
    ccc = c[0] * (gamag - 1) * eg * (pinf * gamap)
    pg = (-bbb + np.sqrt(bbb * bbb + 4 * ccc)) * 0.5
    phig = c[0] * (gamag - 1) * eg / pg
    rog = c[0] / phig
    tg = pg / (rog * R_GAS)
    return np.stack([ug, vg, wg, pg, tg, rog])


@dataclass
class CaseSpec:
    name: str
    mesh: MeshArrays
    flow: dict
    cu: np.ndarray
    ghost_prims: np.ndarray
    steps: int
    extra: dict

    def params(self, **over):
        d = dict(self.flow)
        d.update(self.extra)
        d.update(over)
        return make_params(d)


def shock_bubble(n=20, jitter=0.1, seed=0, radius=0.2, p_post=1.0e9, rho_post=1230.0,
                 center=(0.5, 0.5, 0.5), shock_x=0.2, pinf=6.0e8, gamap=4.4, cpp=4186.0,
                 post_velocity=None, reference_scheme=False, alpha_min=1e-6) -> CaseSpec:
    """Air-water shock-bubble in a closed unit box of n^3 hexes (6 tets each),
    slip walls.  Water at 1e5 Pa / 1000 kg/m^3 ahead of a planar shock at
    x = shock_x, p_post / rho_post behind it; an air bubble (alpha_air =
    1 - 1e-6, 1e5 Pa, 1.2 kg/m^3) of `radius` at `center`; alpha_air = 1e-6
    elsewhere.  The post-shock water moves with the Rankine-Hugoniot velocity
    of that jump unless post_velocity is given."""
    b = box_mesh(n, n, n, jitter=jitter, seed=seed, bc_type=5)
    return shock_bubble_on(b, radius=radius, p_post=p_post, rho_post=rho_post, center=center, shock_x=shock_x,
                           pinf=pinf, gamap=gamap, cpp=cpp, post_velocity=post_velocity,
                           reference_scheme=reference_scheme, alpha_min=alpha_min)


def shock_bubble_on(b: Built, radius=0.2, p_post=1.0e9, rho_post=1230.0, center=(0.5, 0.5, 0.5), shock_x=0.2,
                    pinf=6.0e8, gamap=4.4, cpp=4186.0, post_velocity=None, reference_scheme=False,
                    alpha_min=1e-6) -> CaseSpec:
    """The shock-bubble state of shock_bubble() on an already built unit-box
    mesh (several cases may share one mesh)."""
    gamag = 1.4
    p0, rho0 = 1.0e5, 1000.0
    if post_velocity is None:
        m2 = (p_post - p0) / (1.0 / rho0 - 1.0 / rho_post)
        m = np.sqrt(m2)
        post_velocity = m / rho0 - m / rho_post
    xc = b.xc
    inb = np.sum((xc - np.asarray(center)) ** 2, axis=1) < radius ** 2
    post = xc[:, 0] < shock_x
    ag = np.where(inb, 1.0 - alpha_min, alpha_min)
    p = np.where(post, p_post, p0)
    rho_p = np.where(post, rho_post, rho0)
    t_air = p0 / (1.2 * R_GAS)
    rho_g = p / (R_GAS * t_air)
    u = np.zeros((xc.shape[0], 3))
    u[post, 0] = post_velocity
    cu = conserved(ag, p, rho_g, rho_p, u, gamag, gamap, pinf)
    gp = ghost_prims_from_parents(b.mesh, cu, gamag, gamap, pinf)
    tp0 = (p0 + pinf) * gamap / ((gamap - 1) * rho0 * cpp)
    flow = dict(pmax=p0, pmin=p0, tgmax=t_air, tgmin=t_air, ugmax=0.0, ugmin=0.0, vgmax=0.0, vgmin=0.0,
                wgmax=0.0, wgmin=0.0, upmax=0.0, upmin=0.0, vpmax=0.0, vpmin=0.0, wpmax=0.0, wpmin=0.0,
                tpmax=tp0, tpmin=tp0, pinf=pinf, gamap=gamap, gamag=gamag, cpp=cpp, cpg=1004.5,
                amolg=28.9, prg=0.72, epslnmax=1.0e-3, epslnmin=1.0e-8, epslninf=2.0e-8, phipzero=1.0e-8,
                cfl=0.4, niter=1, itersub=100, istart=1, diap=1.0e-4, surfacetension=0.0, myflux=2,
                myorder=2, as_=1.716e-5 * (1 + 110.4 / 273.15) / np.sqrt(273.15), ts=110.4)
    extra = dict(venkat_k=0.3, rk_scheme=0, inviscid=0) if reference_scheme else \
        dict(venkat_k=5.0, rk_scheme=1, inviscid=1)
    return CaseSpec("shock_bubble", b.mesh, flow, cu, gp, 100, extra)


def cylinder(nr=160, nt=256, nz=20, ndrop=32, seed=1, mach=0.3, re_d=150.0, t_inf=288.15,
             p_inf=101325.0, pinf=6.0e8, gamap=4.4, cpp=4186.0, drop_r=0.1,
             alpha_w_drop=1.0 - 1e-6, alpha_w_bg=1e-6) -> CaseSpec:
    """Viscous air flow past a cylinder (D = 1) on an O-grid to 20D with 32
    water droplets of radius 0.1D (alpha_w = 1 - 1e-6 inside, 1e-6 outside)
    placed uniformly in x in [-8,-3], |y| < 2 (seeded).  Mach 0.3 inflow,
    Re_D through the Sutherland constant, isothermal no-slip wall at the
    free-stream temperature, far field outside."""
    b = ogrid_mesh(nr, nt, nz, seed=seed)
    return _cylinder_flow(b, "cylinder", ndrop=ndrop, seed=seed, mach=mach, re_d=re_d, t_inf=t_inf, p_inf=p_inf,
                          pinf=pinf, gamap=gamap, cpp=cpp, drop_r=drop_r, alpha_w_drop=alpha_w_drop,
                          alpha_w_bg=alpha_w_bg)


def _cylinder_flow(b: Built, name, ndrop=32, seed=1, mach=0.3, re_d=150.0, t_inf=288.15, p_inf=101325.0,
                   pinf=6.0e8, gamap=4.4, cpp=4186.0, drop_r=0.1, alpha_w_drop=1.0 - 1e-6,
                   alpha_w_bg=1e-6) -> CaseSpec:
    """Initial state and parameters of the cylinder flow on mesh b."""
    gamag = 1.4
    a_inf = np.sqrt(gamag * R_GAS * t_inf)
    U = mach * a_inf
    rho_inf = p_inf / (R_GAS * t_inf)
    mu = rho_inf * U * 1.0 / re_d
    ts = 110.4
    as_ = mu * (1 + ts / t_inf) / np.sqrt(t_inf)
    rng = np.random.default_rng(seed)
    dc = np.stack([rng.uniform(-8, -3, ndrop), rng.uniform(-2, 2, ndrop),
                   rng.uniform(drop_r, 4.0 - drop_r, ndrop)], axis=1)
    xc = b.xc
    inside = np.zeros(xc.shape[0], bool)
    for c in dc:
        inside |= np.sum((xc - c) ** 2, axis=1) < drop_r ** 2
    ag = np.where(inside, 1.0 - alpha_w_drop, 1.0 - alpha_w_bg)
    p = np.full(xc.shape[0], p_inf)
    u = np.zeros((xc.shape[0], 3))
    u[:, 0] = U
    rho_g = np.full(xc.shape[0], rho_inf)
    rho_p = np.full(xc.shape[0], 1000.0)
    cu = conserved(ag, p, rho_g, rho_p, u, gamag, gamap, pinf)
    gp = ghost_prims_from_parents(b.mesh, cu, gamag, gamap, pinf)
    tp = (p_inf + pinf) * gamap / ((gamap - 1) * 1000.0 * cpp)
    flow = dict(pmax=p_inf, pmin=p_inf, tgmax=t_inf, tgmin=t_inf, ugmax=U, ugmin=U, vgmax=0.0, vgmin=0.0,
                wgmax=0.0, wgmin=0.0, upmax=U, upmin=U, vpmax=0.0, vpmin=0.0, wpmax=0.0, wpmin=0.0,
                tpmax=tp, tpmin=tp, pinf=pinf, gamap=gamap, gamag=gamag, cpp=cpp, cpg=1004.5,
                amolg=28.9, prg=0.72, epslnmax=1.0e-3, epslnmin=1.0e-8, epslninf=2.0e-8, phipzero=1.0e-6,
                cfl=0.5, niter=1, itersub=1000, istart=1, diap=1.0e-4, surfacetension=0.0, myflux=2,
                myorder=2, as_=as_, ts=ts)
    extra = dict(venkat_k=5.0, rk_scheme=1, inviscid=0, twall=t_inf)
    return CaseSpec(name, b.mesh, flow, cu, gp, 1000, extra)


def with_dispersed(spec: CaseSpec, fractions=(2.0e-3, 1.0e-3, 5.0e-4), rho=(2500.0, 1950.0, 2700.0),
                   rad=(5.0e-6, 20.0e-6, 7.5e-6), slip=0.02) -> CaseSpec:
    """The five-phase form of a two-phase case: three dispersed phases q, r,
    s (particles of density rho and radius rad, the reference's FIVE_PHASE
    model, flow.in groups 19-20) whose volume fractions vary smoothly around
    `fractions` over the domain, moving with the liquid velocity plus a small
    slip (so their drag is not zero).  The gas and liquid fractions are
    scaled by the volume left to them, so the five fractions sum to one and
    the pressure recovered by the five-phase equation of state is the case's
    own.  Variables 11-22 of cu: mass and momentum of q, r, s."""
    m = spec.mesh
    el = m.elem[:, :4] - 1
    xc = np.stack([m.x[el].mean(1), m.y[el].mean(1), m.z[el].mean(1)], axis=1)
    lo, hi = xc.min(axis=0), xc.max(axis=0)
    t = (xc - lo) / np.maximum(hi - lo, 1e-30)
    phd = [f * (1.0 + 0.5 * np.sin(2 * np.pi * (k + 1) * t[:, k % 3]) * np.cos(np.pi * t[:, (k + 1) % 3]))
           for k, f in enumerate(fractions)]
    aaa = 1.0 - phd[0] - phd[1] - phd[2]
    cu2 = spec.cu.copy() * aaa[None, :]
    up = cu2[6:9] / cu2[5][None, :]
    cu = np.empty((22, m.neles))
    cu[:10] = cu2
    for d in range(3):
        ud = up * (1.0 + slip * (d + 1))
        cu[10 + 4 * d] = phd[d] * rho[d]
        cu[11 + 4 * d:14 + 4 * d] = (phd[d] * rho[d])[None, :] * ud
    flow = dict(spec.flow, rhoq=rho[0], rhor=rho[1], rhos=rho[2], radq=rad[0], radr=rad[1], rads=rad[2],
                phiqinit=fractions[0], phirinit=fractions[1], phisinit=fractions[2])
    return CaseSpec(spec.name + "_five_phase", m, flow, cu, spec.ghost_prims, spec.steps,
                    dict(spec.extra, five_phase=1))


def union_mesh(a: Built, b: Built) -> tuple[Built, np.ndarray]:
    """One element list of two meshes: a's elements, then b's; ghosts of a,
    then of b, all after the elements (so no ghost id aliases an element id,
    unlike meshes merged without ghost offsets).  Returns the union and the
    block of each element (0 for a, 1 for b)."""
    ma, mb = a.mesh, b.mesh
    ea, eb, ga = ma.neles, mb.neles, ma.nghosts
    E = ea + eb

    def remap(nc, ne_own, eoff, goff):
        out = nc.astype(np.int64).copy()
        el = nc <= ne_own
        out[el] = nc[el] + eoff
        out[~el] = E + goff + (nc[~el] - ne_own)
        return out

    el_a, el_b = ma.elem.copy(), mb.elem.copy()
    el_b[:, 0:4] += ma.nodes
    el_a[:, 4:8] = remap(ma.elem[:, 4:8], ea, 0, 0)
    el_b[:, 4:8] = remap(mb.elem[:, 4:8], eb, ea, ga)
    gh_a, gh_b = ma.ghost.copy(), mb.ghost.copy()
    gh_a[:, 1] = E + (ma.ghost[:, 1] - ea)
    gh_b[:, 0] += ea
    gh_b[:, 1] = E + ga + (mb.ghost[:, 1] - eb)
    mesh = MeshArrays(np.concatenate([ma.x, mb.x]), np.concatenate([ma.y, mb.y]), np.concatenate([ma.z, mb.z]),
                      np.concatenate([el_a, el_b]).astype(np.int32), np.concatenate([gh_a, gh_b]).astype(np.int32))
    block = np.concatenate([np.zeros(ea, np.int32), np.ones(eb, np.int32)])
    return Built(mesh, np.concatenate([a.xc, b.xc]), np.concatenate([a.vol, b.vol])), block


@dataclass
class OversetSpec:
    """An overset case: the union mesh with the hole cut as iblank 0, the
    block of each element and the component's outer boundary type."""
    spec: CaseSpec
    block: np.ndarray
    outer_type: int
    layers: int


def overset_cylinder(bg=(200, 120, 20), comp=(96, 256, 20), hole_r=1.2, comp_r_out=3.0, layers=2, seed=1,
                     box=((-10.0, -12.0, 0.0), (30.0, 12.0, 4.0)), hole_cut="radius", **flow_kw) -> OversetSpec:
    """Overset cylinder: a background box of bg hexes on [-10,30]x[-12,12]x[0,4]
    (6 tets each; far field on its x/y faces, symmetry 53 on z; `box` moves
    its corners, the span must stay [0, 4]) and an O-grid
    component of comp = (radial, azimuthal, spanwise) hexes around the
    cylinder (D = 1) out to comp_r_out; background cells whose centroid lies
    within hole_r of the cylinder axis are holes (iblank 0).  hole_cut="wall"
    cuts them with the library instead (hp_overset_hole_cut: within
    hole_r - 0.5 of the cylinder's wall faces, or inside them), which differs
    from the radius rule only within the polygonal wall's deviation from the
    circle.  Flow as in cylinder() (Mach 0.3, Re_D 150, droplets)."""
    nx, ny, nz = bg

    def bg_types(fc):
        t = np.full(fc.shape[0], 7)
        t[(fc[:, 2] < 1e-9) | (fc[:, 2] > 4.0 - 1e-9)] = 53
        return t

    a = box_mesh(nx, ny, nz, lo=box[0], hi=box[1], seed=seed, bc_type=bg_types)
    nr, nt, nzc = comp
    b = ogrid_mesh(nr, nt, nzc, r_in=0.5, r_out=comp_r_out, dr0=0.005, seed=seed + 1)
    u, block = union_mesh(a, b)
    if hole_cut == "wall":
        from .engine import overset_hole_cut
        u.mesh.elem[:, 8], _ = overset_hole_cut(u.mesh, block, wall_type=6, margin=hole_r - 0.5)
    elif hole_cut == "radius":
        hole = (block == 0) & (np.hypot(u.xc[:, 0], u.xc[:, 1]) < hole_r)
        u.mesh.elem[hole, 8] = 0
    else:
        raise ValueError(f"hole_cut must be 'radius' or 'wall', not {hole_cut!r}")
    spec = _cylinder_flow(u, "overset_cylinder", seed=seed, **flow_kw)
    return OversetSpec(spec, block, 7, layers)


# ---------------------------------------------------------------------------
FLOW_TEMPLATE = """# Pressure limits
{pmax!r}    {pmin!r}   # pmax, pmin
# Gas temperature limits
{tgmax!r}     {tgmin!r}    # tgmax, tgmin
# Velocity limits (x, y, z components)
{ugmax!r}     {ugmin!r}  # ugmax, ugmin
{vgmax!r}     {vgmin!r}  # vgmax, vgmin
{wgmax!r}     {wgmin!r}  # wgmax, wgmin
# Particle velocity limits (x, y, z components)
{upmax!r}     {upmin!r}  # upmax, upmin
{vpmax!r}     {vpmin!r}  # vpmax, vpmin
{wpmax!r}     {wpmin!r}  # wpmax, wpmin
# Particle temperature limits
{tpmax!r}     {tpmin!r}  # tpmax, tpmin
# Reference pressure, specific heat ratios, and properties
{pinf!r}   {gamap!r}   # pinf, gamap
{gamag!r}   {cpp!r}   # gamag, cpp
{cpg!r}   {amolg!r}   # cpg, amolg
{prg!r}   {epslnmax!r}   # prg, epslnmax
# Solver settings
{epslnmin!r}   {epslninf!r}   {phipzero!r} # epslnmin, epslninf , phipdrop
{cfl!r}  {niter}    {itersub} # cfl, niter, itersub
{istart}     {diap!r}     # istart, diap
{surfacetension!r}   {myflux}       # surfacetension, myflux
{myorder}   {as_!r}   {ts!r}   # myorder, as, ts
"""


def write_case_dir(spec: CaseSpec, path: str) -> None:
    """Write a case directory the reference (and this engine's readers)
    accept: flow.in, itter.in, geometry_files/*, restart_files/restart0000.in."""
    from .engine import write_restart
    os.makedirs(os.path.join(path, "geometry_files"), exist_ok=True)
    os.makedirs(os.path.join(path, "restart_files"), exist_ok=True)
    fl = {k: (float(v) if isinstance(v, (float, np.floating)) else v) for k, v in spec.flow.items()}
    with open(os.path.join(path, "flow.in"), "w") as f:
        f.write(FLOW_TEMPLATE.format(**fl))
    with open(os.path.join(path, "itter.in"), "w") as f:
        f.write("           0\n")
    m = spec.mesh
    with open(os.path.join(path, "geometry_files", "grid_proc0000.dat"), "w") as f:
        f.write(f"{m.nodes:12d}{m.neles:12d}\n")
        ids = np.arange(1, m.nodes + 1)
        nd = np.column_stack([ids, m.x, m.y, m.z, np.ones(m.nodes), np.ones(m.nodes)])
        np.savetxt(f, nd, fmt="%12d %25.17E %25.17E %25.17E %12d %12d")
        el = np.column_stack([np.arange(1, m.neles + 1), m.elem])
        np.savetxt(f, el, fmt="%12d")
    with open(os.path.join(path, "geometry_files", "bc_proc0000.in"), "w") as f:
        f.write(f"{m.nghosts:12d}\n")
        np.savetxt(f, m.ghost, fmt="%12d")
    with open(os.path.join(path, "geometry_files", "proc_bc0000.in"), "w") as f:
        f.write("           0           0\n")
    write_restart(os.path.join(path, "restart_files", "restart0000.in"), 0.0, spec.cu, spec.ghost_prims)


@dataclass
class StreamCase:
    """One request of a serving stream: arrival time (s from the stream's
    start), number of steps, and the case itself."""
    rid: int
    arrival: float
    steps: int
    spec: CaseSpec


def serving_stream(n_cases=256, rate=40.0, steps=500, cells=(6000, 400000), seed=2, alpha_min=0.1,
                   jitter=0.1, cfl=0.05):
    """A stream of shock-bubble cases: mesh sizes log-uniform in `cells`
    (box grids of n^3 hexes split into 6 tets, n = round((cells/6)^(1/3)),
    jittered by +-jitter*h), bubble radius U[0.1, 0.3], post-shock water
    pressure log-U[1e8, 2e9] Pa, Poisson arrivals at `rate` per second, all
    drawn from `seed`.  Cases of the same n share one mesh (its generation is
    the client's cost, not the server's); each carries its own state.  The
    explicit scheme keeps these cases finite over 500 SSP-RK3 steps at CFL
    0.05 with an air volume fraction of 1 - alpha_min / alpha_min, on every
    mesh size of the stream (at CFL 0.1 the finest meshes blow up after
    200-400 steps, at CFL 0.4 within 25-100 steps, and at alpha_min = 1e-6 at
    any CFL)."""
    rng = np.random.default_rng(seed)
    target = np.exp(rng.uniform(np.log(cells[0]), np.log(cells[1]), n_cases))
    nside = np.maximum(np.rint(np.cbrt(target / 6.0)).astype(int), 2)
    radius = rng.uniform(0.1, 0.3, n_cases)
    p_post = np.exp(rng.uniform(np.log(1.0e8), np.log(2.0e9), n_cases))
    gaps = rng.exponential(1.0 / rate, n_cases)
    arrival = np.cumsum(gaps) - gaps[0]
    meshes = {}
    out = []
    for k in range(n_cases):
        n = int(nside[k])
        if n not in meshes:
            meshes[n] = box_mesh(n, n, n, jitter=jitter, seed=1000 * seed + n, bc_type=5)
        spec = shock_bubble_on(meshes[n], radius=float(radius[k]), p_post=float(p_post[k]), alpha_min=alpha_min)
        spec.flow["cfl"] = cfl
        out.append(StreamCase(k, float(arrival[k]), int(steps), spec))
    return out


def shock_lattice(nx=60, ny=60, nz=90, jitter=0.15, seed=3, p_post=5.0e9, lattice=5, radius=0.05,
                  shock_z=0.2, bubble_z=0.5, alpha_min=0.1, cfl=0.05, pinf=6.0e8, gamap=4.4,
                  cpp=4186.0) -> CaseSpec:
    """Precision stress: a planar water shock (p_post behind it, 1e5 Pa ahead:
    a pressure ratio of 5e4 at 5e9 Pa) travelling in +z through a box of
    nx x ny x nz hexes (6 tets each) on [0,1] x [0,1] x [0, nz/nx], jittered
    by +-jitter*h, towards a lattice x lattice grid of air bubbles of
    `radius` in the plane z = bubble_z.  Slip walls; SSP-RK3, K = 5,
    inviscid; air volume fraction 1 - alpha_min in the bubbles, alpha_min
    outside (the stable contrast of this scheme, as in serving_stream)."""
    b = box_mesh(nx, ny, nz, hi=(1.0, 1.0, nz / nx), jitter=jitter, seed=seed, bc_type=5)
    gamag = 1.4
    p0, rho0 = 1.0e5, 1000.0
    rho_post = rho0 * (1.0 + (p_post - p0) / (gamap * (p0 + pinf)))   # weak-shock estimate of the
    rho_post = min(rho_post, 1.8 * rho0)                              # jump, capped at 1.8x
    m2 = (p_post - p0) / (1.0 / rho0 - 1.0 / rho_post)
    post_velocity = np.sqrt(m2) / rho0 - np.sqrt(m2) / rho_post
    xc = b.xc
    cen = (np.arange(lattice) + 0.5) / lattice
    inb = np.zeros(xc.shape[0], bool)
    for cx in cen:
        for cy in cen:
            inb |= (xc[:, 0] - cx) ** 2 + (xc[:, 1] - cy) ** 2 + (xc[:, 2] - bubble_z) ** 2 < radius ** 2
    post = xc[:, 2] < shock_z
    ag = np.where(inb, 1.0 - alpha_min, alpha_min)
    p = np.where(post, p_post, p0)
    rho_p = np.where(post, rho_post, rho0)
    t_air = p0 / (1.2 * R_GAS)
    rho_g = p / (R_GAS * t_air)
    u = np.zeros((xc.shape[0], 3))
    u[post, 2] = post_velocity
    cu = conserved(ag, p, rho_g, rho_p, u, gamag, gamap, pinf)
    gp = ghost_prims_from_parents(b.mesh, cu, gamag, gamap, pinf)
    spec = shock_bubble_on(b, alpha_min=alpha_min)      # parameters of the shock-bubble family
    spec.name = "shock_lattice"
    spec.cu, spec.ghost_prims = cu, gp
    spec.flow["cfl"] = cfl
    spec.steps = 2000
    return spec
