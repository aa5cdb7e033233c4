"""Generate the golden fixtures of tests/golden/ by running the reference CoMech code itself.

Run where the reference checkout is readable, naming its root in COMECH_REF:

    COMECH_REF=<path to the CoMech checkout> python tests/golden/make_golden.py

Every fixture stores its inputs as well as the reference's outputs, so the tests never need the
reference (nor the synthetic generator) at run time.  Reference functions used:
fe/solver.py (element_matrices, element_basis, Grid, assemble, solve, cell_stress),
fe/gmg.py (GMG, pcg_gmg), rb/splitfe.py (split_connectivity[_fast], KL_family, assemble_cn,
solve_cn, cell_stress_cn, element_forces_cn), fe/test_patch.py (patch-test set-up),
rb/rbsim.py (rigid_fit, sample_fe, sample_nodes) and the region-force sums of rb/rbfe.py:194-213.

    COMECH_REF=... python tests/golden/make_golden.py [fixture ...]      # default: all fixtures
"""
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("COMECH_REF")
if not REF:
    sys.exit("make_golden.py: set COMECH_REF to the root of the reference CoMech checkout")
sys.path.insert(0, REPO)
sys.path.insert(1, REF)
sys.path.insert(2, os.path.join(REF, "rb"))

from fe import solver as RS          # noqa: E402  (reference)
from fe import gmg as RG             # noqa: E402
import splitfe as RSF                # noqa: E402
from comech_b200 import synth        # noqa: E402  (input generator only)


def save(name, **arrs):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print("wrote", name, {k: np.shape(v) for k, v in arrs.items()})


def springs_arrays(s):
    return dict(pair_a=s.pair_a, pair_b=s.pair_b, pair_k=s.pair_k, line_a=s.line_a, line_b=s.line_b,
                line_d=s.line_d, line_k=s.line_k)


def elements():
    out = {}
    for i, d in enumerate([(1.0, 1.0, 1.0), (0.5, 0.75, 1.25), (3.0, 1.5, 0.3)]):
        KL, KM, Bc = RS.element_matrices(np.array(d))
        out[f"dims{i}"] = np.array(d); out[f"KL{i}"] = KL; out[f"KM{i}"] = KM; out[f"Bc{i}"] = Bc
        out[f"KB{i}"] = RS.element_basis(np.array(d))
    g = RS.Grid(np.r_[0, 1, 3, 4, 7, 10], np.r_[0, 2, 5, 10], np.r_[0, 1, 2, 4, 6, 10])
    out["patch_KLsri"] = RSF.KL_family(g)
    out["patch_udims"] = g.udims
    out["patch_dim_id"] = g.dim_id
    out["patch_cell_nodes"] = g.cell_nodes
    out["patch_node_xyz"] = g.node_xyz
    save("elements", **out)


def split_cases():
    out = {}
    P = synth.hindfoot_problem(28, 20, 16, h=2.8, seed=3)
    g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    cn, orig, ns = RSF.split_connectivity_fast(g, P["active"], P["part"], P["bone_share"])
    cn2, orig2, ns2 = RSF.split_connectivity(g, P["active"], P["part"], P["bone_share"])
    assert (cn == cn2).all() and (orig == orig2).all() and ns == ns2
    out.update(h_edges_x=g.xe, h_edges_y=g.ye, h_edges_z=g.ze, h_active=P["active"], h_part=P["part"],
               h_share=P["bone_share"], h_cn=cn, h_orig=orig, h_nsplit=ns)
    # random parts and shares: many bones, ties in share and in cell counts
    rng = np.random.default_rng(11)
    g2 = RS.Grid(np.arange(13.0), np.arange(11.0), np.arange(9.0))
    act = rng.random(g2.ncell) < 0.9
    part = rng.integers(0, 5, g2.ncell) * (rng.random(g2.ncell) < 0.7)
    share = np.round(rng.random((g2.ncell, 5)) * 4) / 4 * (rng.random((g2.ncell, 5)) < 0.5)
    share[:, 0] = 0
    cn, orig, ns = RSF.split_connectivity_fast(g2, act, part, share)
    cn2, orig2, ns2 = RSF.split_connectivity(g2, act, part, share)
    assert (cn == cn2).all() and (orig == orig2).all() and ns == ns2
    out.update(r_edges_x=g2.xe, r_edges_y=g2.ye, r_edges_z=g2.ze, r_active=act, r_part=part, r_share=share,
               r_cn=cn, r_orig=orig, r_nsplit=ns)
    save("split", **out)


def hindfoot_solve():
    P = synth.hindfoot_problem(24, 18, 16, h=3.0, seed=1)
    g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    cells = np.flatnonzero(P["active"])
    K, nmap, nused = RSF.assemble_cn(g, P["lam"], P["mu"], cells, P["cn"])
    rng = np.random.default_rng(5)
    u = rng.standard_normal((2, K.shape[0]))
    Ku = np.stack([K @ x for x in u])
    U, info, R = RSF.solve_cn(g, P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"],
                              P["extra"], P["node_groups"], tol=1e-10, maxiter=800)
    sig, vm, eps = RSF.cell_stress_cn(g, P["lam"], P["mu"], U, cells, P["cn"])
    fcells = cells[::7]
    F = RSF.element_forces_cn(g, P["lam"], P["mu"], U, fcells, P["cn"])
    (ln, la, lt), = P["loads"]
    groups = np.concatenate(P["node_groups"]); glen = np.array([len(x) for x in P["node_groups"]])
    save("hindfoot_small", xe=g.xe, ye=g.ye, ze=g.ze, lam=P["lam"], mu=P["mu"], active=P["active"], cn=P["cn"],
         orig=P["orig"], fixed_nodes=P["fixed"][0], fixed_area=P["fixed"][1], load_nodes=ln, load_area=la,
         load_t=lt, groups=groups, group_len=glen, nused=nused, u=u, Ku=Ku, U=U, R=R, iters=info["iters"],
         flag=info["flag"], levels=info["levels"], ndof=info["ndof"], sig=sig, vm=vm, eps=eps, fcells=fcells, F=F,
         **springs_arrays(P["extra"]))
    # multigrid internals on the assembled operator of this problem
    kd = np.zeros(K.shape[0])
    for c in range(3):
        np.add.at(kd, 3 * nmap[P["fixed"][0]] + c, P["fixed"][1] * 1e6)
    A = K + RS.sp.diags(kd) + P["extra"](nmap, K.shape[0])
    mg = RG.GMG(A.tocsr(), P["orig"][nused], g.xe, g.ye, g.ze, min_dofs=600)
    b = rng.standard_normal(A.shape[0])
    save("gmg_small", nused=nused, b=b, vcycle=mg.vcycle(b), sizes=np.array([L.A.shape[0] for L in mg.levels]),
         lmax=np.array([L.lmax for L in mg.levels]))


def region_forces_ref(g, lam, mu, U, cn, active, part, lab, nlab, target):
    """The force sums of rb/rbfe.py:199-213 (inline there) for one target part, per label."""
    cells = np.arange(g.ncell)
    tgt = (part == target) & active
    tn = np.zeros(len(U), bool)
    tn[cn[cells[tgt]].ravel()] = True
    oc = cells[active & ~tgt]
    oc = oc[tn[cn[oc]].any(1)]
    fe = RSF.element_forces_cn(g, lam, mu, U, oc, cn)
    fsum = -(fe * tn[cn[oc]][:, :, None]).sum(1)
    out = np.zeros((nlab, 3))
    present = np.zeros(nlab, bool)
    for i in range(nlab):
        m = lab[oc] == i
        if m.any():
            out[i] = fsum[m].sum(0)
            present[i] = True
    return out, present


def post():
    """Post-processing of the hindfoot_small solution: region forces on two bones, rigid fit of a bone and the
    displacement relative to it, resampling on an analysis grid that sticks out of the FE grid."""
    sys.path.insert(0, os.path.join(REF, "rb"))
    import rbsim as RB                   # noqa: E402
    P = synth.hindfoot_problem(24, 18, 16, h=3.0, seed=1)
    g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    U, info, R = RSF.solve_cn(g, P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"],
                              P["extra"], P["node_groups"], tol=1e-10, maxiter=800)
    cells = np.flatnonzero(P["active"])
    sig, vm, eps = RSF.cell_stress_cn(g, P["lam"], P["mu"], U, cells, P["cn"])
    VM = np.zeros(g.ncell, np.float32); VM[cells] = vm
    SIG = np.zeros((g.ncell, 6), np.float32); SIG[cells] = sig
    rng = np.random.default_rng(21)
    nlab = 7
    lab = rng.integers(0, nlab, g.ncell).astype(np.int32)
    part = P["part"].astype(np.int32)
    out = dict(xe=g.xe, ye=g.ye, ze=g.ze, lam=P["lam"], mu=P["mu"], active=P["active"], cn=P["cn"], orig=P["orig"],
               U=U, VM=VM, SIG=SIG, lab=lab, part=part, nlab=nlab)
    for target in (1, 2):
        F, pres = region_forces_ref(g, P["lam"], P["mu"], U, P["cn"], P["active"], part, lab, nlab, target)
        out[f"F{target}"] = F
        out[f"present{target}"] = pres
    xyz = g.node_xyz[P["orig"]]
    nodes = np.unique(P["cn"][cells[part[cells] == 1]].ravel())
    t, w, c = RB.rigid_fit(xyz[nodes], np.nan_to_num(U[nodes]))
    Urel = np.nan_to_num(U) - (t[None, :] + np.cross(w[None, :], xyz - c[None, :]))
    out.update(fit_nodes=nodes, fit_t=t, fit_w=w, fit_c=c, Urel=Urel)
    gm = RS.Grid(np.arange(-4.0, 80.0, 5.0), np.arange(-3.0, 60.0, 5.0), np.arange(2.0, 52.0, 5.0))
    o = dict(g=g, cn=P["cn"], active=P["active"], VM=VM, SIG=SIG)
    vm_c, u_c, frac = RB.sample_fe(o, gm, Urel, sub=2)
    out.update(ml_xe=gm.xe, ml_ye=gm.ye, ml_ze=gm.ze, vm_c=vm_c, u_c=u_c, frac=frac, sig_c=RB.sample_fe.sig)
    out["u_nodes"] = RB.sample_nodes(o, gm, Urel)
    save("post", **out)


def materials_case():
    """Material mixing of rb/rbfe.py:75-134 on a seeded sub-voxel label raster: bone bodies of the atlas
    roles (cortical / cancellous), joint cartilages, coalition / fibrous / fat / fusion / gap bodies, soft
    tissue and fascia, in blobs so that joint cells (two bone groups within one cell) occur."""
    sys.path.insert(0, os.path.join(REF, "rb"))
    import rbfe as RF                    # noqa: E402
    import rbgeom as RG                  # noqa: E402
    rng = np.random.default_rng(31)
    nx, ny, nz, ns = 14, 11, 9, 3
    bodies = [1, 53, 2, 52, 40, 45, 43, 49, 3, 54, 4, 13, 70, 71] + list(RG.CART.values()) + \
        [RG.SOFT, RG.FASCIA, RG.COAL, RG.FIB, RG.INTERP, RG.FUSE, RG.GAP]
    cls = {1: 1, 53: 2, 2: 1, 52: 2, 40: 1, 45: 2, 43: 1, 49: 2, 3: 1, 54: 2, 4: 1, 13: 2, 70: 1, 71: 2,
           RG.SOFT: 5, RG.FASCIA: 4, RG.COAL: 1, RG.FIB: 7, RG.INTERP: 8, RG.FUSE: 1, RG.GAP: 9}
    for c in RG.CART.values():
        cls[c] = 3
    # blobs on the sub-voxel grid, void elsewhere
    sx, sy, sz = nx * ns, ny * ns, nz * ns
    lab = np.zeros((sx, sy, sz), np.int64)
    X, Y, Z = np.meshgrid(np.arange(sx), np.arange(sy), np.arange(sz), indexing="ij")
    for _ in range(60):
        b = bodies[rng.integers(len(bodies))]
        c = rng.uniform(0, 1, 3) * (sx, sy, sz)
        r = rng.uniform(2, 9)
        lab[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 < r * r] = b
    # cell sample order: cell id (z fastest), then the sub-voxels (z fastest)
    L = lab.reshape(nx, ns, ny, ns, nz, ns).transpose(0, 2, 4, 1, 3, 5).reshape(nx * ny * nz, ns ** 3)
    V = dict(cls={str(k): v for k, v in cls.items()}, L=L, xe=np.arange(nx + 1.0), ye=np.arange(ny + 1.0),
             ze=np.arange(nz + 1.0))
    out = dict(L=L, nx=nx, ny=ny, nz=nz, cls_body=np.array(sorted(cls)), cls_class=np.array([cls[b] for b in sorted(cls)]))
    for name, kw in (("a", {}), ("b", dict(cart_E=3.0, nu_soft=0.45))):
        E, nu, active, F, ser = RF.materials(V, RF.ROLES, **kw)
        out.update({f"{name}_E": E, f"{name}_nu": nu, f"{name}_active": active, f"{name}_F": F, f"{name}_ser": ser})
    out["b_cart_E"] = 3.0
    out["b_nu_soft"] = 0.45
    names = list(RF.ROLES["bones"])
    out["role_names"] = np.array(names)
    out["role_len"] = np.array([len(RF.ROLES["bones"][n]) for n in names])
    out["role_bodies"] = np.concatenate([np.array(RF.ROLES["bones"][n]) for n in names])
    out["role_bonded_extra"] = np.array(RF.ROLES["bonded_extra"])
    save("materials", **out)


def block_solves():
    P = synth.block_problem(12, 10, 8, h=1.0, seed=2)
    g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    (sn, sa, sk), = P["springs"]; (ln, la, lt), = P["loads"]
    cells = np.arange(g.ncell)
    out = dict(xe=g.xe, ye=g.ye, ze=g.ze, lam=P["lam"], mu=P["mu"], spring_nodes=sn, spring_area=sa, spring_k=sk,
               load_nodes=ln, load_area=la, load_t=lt)
    U, info = RS.solve(g, P["lam"], P["mu"], P["active"], P["springs"], P["loads"], method="gmg", tol=1e-10)
    sig, vm, eps = RS.cell_stress(g, P["lam"], P["mu"], U, cells)
    out.update(U_gmg=U, iters_gmg=info["iters"], vm_gmg=vm, sig_gmg=sig)
    # rank-1 penalty on the mean x translation of the top face, rigid groups, orthotropic coefficients
    top = cells[g.cK == g.nz - 1]
    tn, ta = RS.face_node_areas(g, top, "z+")
    pen = [(tn, ta, 0, 1e5)]
    coeffs = RS.ortho_coeffs(P["lam"], P["mu"], shear_factor=0.5)
    half = np.unique(g.cell_nodes[cells[g.cI < g.nx // 2]])
    U2, info2 = RS.solve(g, P["lam"], P["mu"], P["active"], P["springs"], P["loads"], method="gmg", tol=1e-10,
                         penalties=pen, coeffs=coeffs, node_groups=[half])
    sig2, vm2, eps2 = RS.cell_stress(g, P["lam"], P["mu"], U2, cells, coeffs=coeffs)
    out.update(pen_nodes=tn, pen_w=ta, pen_comp=0, pen_k=1e5, coeffs=coeffs, group=half, U_pen=U2,
               iters_pen=info2["iters"], vm_pen=vm2, sig_pen=sig2)
    U3, info3 = RS.solve(g, P["lam"], P["mu"], P["active"], P["springs"], P["loads"], method="cg", tol=1e-10)
    out.update(U_cg=U3, iters_cg=info3["iters"])
    save("block_small", **out)


def patch():
    g = RS.Grid(np.r_[0, 1, 3, 4, 7, 10], np.r_[0, 2, 5, 10], np.r_[0, 1, 2, 4, 6, 10])
    E, nu = 1000.0, 0.3
    lam, mu = RS.lame(np.full(g.ncell, E), np.full(g.ncell, nu))
    active = np.ones(g.ncell, bool)
    bot = np.flatnonzero(g.cK == 0); top = np.flatnonzero(g.cK == g.nz - 1)
    nb, ab = RS.face_node_areas(g, bot, "z-"); nt, at = RS.face_node_areas(g, top, "z+")
    U, info = RS.solve(g, lam, mu, active, [(nb, ab, np.array([1e-6, 1e-6, 1e9]))], [(nt, at, np.array([0, 0, -1.0]))],
                       method="direct")
    sig, vm, eps = RS.cell_stress(g, lam, mu, U, np.arange(g.ncell))
    save("patch", xe=g.xe, ye=g.ye, ze=g.ze, E=E, nu=nu, U=U, sig=sig, vm=vm)


# seeded surgical actions of the batch configuration on a mid-size hindfoot (80 x 55 x 47.5 mm at 2.5 mm)
ACTION_CASE = dict(nx=32, ny=22, nz=19, h=2.5, seed=4)


def input_digest(P):
    """Sums of the generator's output that the tests recompute to detect a changed generator."""
    return np.array([P["lam"].sum(), P["mu"].sum(), P["active"].sum(), P["cn"].sum(), len(P["orig"]),
                     P["fixed"][1].sum(), P["loads"][0][1].sum(), P["extra"].node_coo()[4].sum()], float)


def actions():
    """solve_cn of the reference on the instance of each action (rb/splitfe.py:123-158), with stress."""
    out = {}
    for act in ("resection", "osteotomy", "interposition", "fusion", "load"):
        P = synth.hindfoot_problem(ACTION_CASE["nx"], ACTION_CASE["ny"], ACTION_CASE["nz"], h=ACTION_CASE["h"],
                                   seed=ACTION_CASE["seed"], action=act)
        g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
        U, info, R = RSF.solve_cn(g, P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"],
                                  P["extra"], P["node_groups"], tol=1e-10, maxiter=800)
        cells = np.flatnonzero(P["active"])
        sig, vm, eps = RSF.cell_stress_cn(g, P["lam"], P["mu"], U, cells, P["cn"])
        out.update({f"{act}_digest": input_digest(P), f"{act}_U": U, f"{act}_R": R, f"{act}_vm": vm,
                    f"{act}_iters": info["iters"], f"{act}_ndof": info["ndof"]})
    save("actions", case=np.array([ACTION_CASE[k] for k in ("nx", "ny", "nz", "h", "seed")], float), **out)


def spring_hook():
    """The reference's ligament hook (rb/replica3.py:68-86): ends averaged over the bone nodes within
    max(4 mm, the 8th-nearest distance), K += k w w^T per spring, used through solve_cn's extra argument the way
    the engine builds it (rb/rbfe.py:167-179: end bone = the bone nearest to the end point)."""
    import replica3 as R3
    from scipy.spatial import cKDTree
    P = synth.hindfoot_problem(24, 18, 16, h=3.0, seed=3)
    g = RS.Grid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    cn, orig, active, part = P["cn"], P["orig"], P["active"], P["part"]
    cells = np.flatnonzero(active)
    xyz = g.node_xyz[orig]
    names = {1: "talus", 2: "calcaneus", 3: "navicular"}
    allc = np.arange(g.ncell)
    bone_nodes = {nm: np.unique(cn[allc[(part == k) & active]].ravel()) for k, nm in names.items()}
    rng = np.random.default_rng(17)
    springs = []
    for (ka, kb) in ((1, 2), (1, 3), (2, 3), (1, 2), (2, 3), (1, 3)):
        na, nb = bone_nodes[names[ka]], bone_nodes[names[kb]]
        a = xyz[na[rng.integers(len(na))]] + rng.uniform(-1.0, 1.0, 3)
        b = xyz[nb[rng.integers(len(nb))]] + rng.uniform(-1.0, 1.0, 3)
        springs.append(dict(a=a.tolist(), b=b.tolist(), k=float(rng.uniform(50.0, 200.0))))
    trees = {nm: cKDTree(xyz[nd]) for nm, nd in bone_nodes.items() if len(nd)}
    for s_ in springs:
        for key, pt in (("A", s_["a"]), ("B", s_["b"])):
            s_[key] = min(trees, key=lambda nm: trees[nm].query(pt)[0])
    hook = R3.spring_matrix_cn(xyz, springs, bone_nodes)
    U, info, R = RSF.solve_cn(g, P["lam"], P["mu"], active, cn, orig, P["fixed"], P["loads"], hook, P["node_groups"],
                              tol=1e-10, maxiter=800)
    # the hook's matrix on full-layout dofs (3 node + component), for a hook-shaped callable in the tests
    nused = np.unique(cn[cells])
    nmap = -np.ones(len(orig), np.int64)
    nmap[nused] = np.arange(len(nused))
    M = hook(nmap, 3 * len(nused)).tocoo()
    rows = 3 * nused[M.row // 3] + M.row % 3
    cols = 3 * nused[M.col // 3] + M.col % 3
    (ln, la, lt), = P["loads"]
    groups = np.concatenate(P["node_groups"]); glen = np.array([len(x) for x in P["node_groups"]])
    bn = np.concatenate([bone_nodes[names[k]] for k in (1, 2, 3)])
    blen = np.array([len(bone_nodes[names[k]]) for k in (1, 2, 3)])
    save("spring_hook", xe=g.xe, ye=g.ye, ze=g.ze, lam=P["lam"], mu=P["mu"], active=active, cn=cn, orig=orig,
         fixed_nodes=P["fixed"][0], fixed_area=P["fixed"][1], load_nodes=ln, load_area=la, load_t=lt, groups=groups,
         group_len=glen, bone_nodes=bn, bone_len=blen,
         spring_a=np.array([s_["a"] for s_ in springs]), spring_b=np.array([s_["b"] for s_ in springs]),
         spring_k=np.array([s_["k"] for s_ in springs]),
         spring_ends=np.array([[list(names.values()).index(s_["A"]), list(names.values()).index(s_["B"])]
                               for s_ in springs]),
         hook_rows=rows, hook_cols=cols, hook_vals=M.data, U=U, R=R, iters=info["iters"], ndof=info["ndof"])


from label_cases import LABEL_CASES   # noqa: E402  (shared with the tests)



def labels():
    """label_lattice (rb/rbgeom.py:493-524) on seeded synthetic templates (comech_b200.synth.synthetic_template)
    for feet and actions that exercise every branch of label_points; the template is handed to the reference as
    an rbgeom.Template carrying the generated fields."""
    import rbgeom as RB
    from comech_b200 import labels as LB
    out = {}
    for seed in (0, 1):
        T = synth.synthetic_template(seed)
        RT = object.__new__(RB.Template)
        for k in ("lab", "o", "h", "dt", "dc", "so", "facets", "c0", "z_ref", "x_w0", "x_w1", "x_cut0", "z_cut0",
                  "cut_slope", "z_frag_top", "static_bodies"):
            setattr(RT, k, getattr(T, k))
        rng = np.random.default_rng(50 + seed)
        # a whole-foot lattice and a fine lattice over the joint, offset from the raster
        hx = 1.3 + 0.1 * seed
        lat = {"foot": (np.arange(-104.0, 14.0, hx) + rng.uniform(0, 1), np.arange(-36.0, 36.0, hx) + rng.uniform(0, 1),
                        np.arange(4.0, 104.0, hx) + rng.uniform(0, 1)),
               "joint": (np.arange(-76.0, -14.0, 0.6) + rng.uniform(0, 0.5), np.arange(-26.0, 26.0, 0.6) + rng.uniform(0, 0.5),
                         np.arange(40.0, 76.0, 0.6) + rng.uniform(0, 0.5))}
        for name, fk, ak, fill in LABEL_CASES:
            foot, act = RB.Foot(**fk), RB.Action(**ak)
            for ln, (sx, sy, sz) in lat.items():
                key = f"s{seed}_{name}_{ln}"
                out[key] = RB.label_lattice(sx, sy, sz, foot, act, T=RT, defect_fill=fill).astype(np.int16)
                if name == "default" or ln == "joint":
                    out[f"s{seed}_{ln}_sx"], out[f"s{seed}_{ln}_sy"], out[f"s{seed}_{ln}_sz"] = sx, sy, sz
        # a few scattered points through label_points itself
        P = np.column_stack([rng.uniform(-80, -10, 4000), rng.uniform(-25, 25, 4000), rng.uniform(35, 80, 4000)])
        out[f"s{seed}_points"] = P
        for name, fk, ak, fill in LABEL_CASES:
            out[f"s{seed}_{name}_pts"] = RB.label_points(P, RB.Foot(**fk), RB.Action(**ak), T=RT, defect_fill=fill)
    save("labels", **out)


if __name__ == "__main__":
    fixtures = dict(elements=elements, split=split_cases, hindfoot=hindfoot_solve, block=block_solves, patch=patch,
                    post=post, materials=materials_case, actions=actions, spring_hook=spring_hook,
                    labels=labels)
    for name in (sys.argv[1:] or list(fixtures)):
        fixtures[name]()
