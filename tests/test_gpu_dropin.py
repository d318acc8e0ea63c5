"""GPU parity of the reference-named entry points (tier 1 and 2) against the
CPU oracle on the same seeded inputs.

Everything except the FFT path is expected to be bit-identical: the kernels
evaluate the reference's expressions in the same order without FMA
contraction, like the oracle.  The FFT path (p2s/s2p/spn/mkp) uses a
different transform algorithm than the oracle and is held to 1e-13/1e-12.
The only transcendental is the level-set mask's sin (<= 2 ulp).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import bit_equal, maxdiff, oracle_grid, rand_field, rel_l2
from vtkmakecompare_b200 import legacy as G
from vtkmakecompare_b200 import workload as W

pytestmark = pytest.mark.gpu

SIZES = [(8, 6, 10), (12, 9, 8), (16, 12, 20)]


def grid(nx, ny, nz, stretched=True):
    g = W.grid_arrays(nx, ny, nz, 2 * np.pi, 2.0, np.pi, y0=-1.0 if stretched else 0.0,
                      gamma=2.0 if stretched else 0.0)
    return g, oracle_grid(g)


def mask(rng, nx, ny, nz):
    cv = np.zeros((nx, ny, nz, 4), order="F")
    c = rng.random((nx, ny, nz))
    c[c < 0.6] = 0.0
    c[c > 0.9] = 1.0
    cv[..., 0] = c
    cv[..., 1:] = rng.random((nx, ny, nz, 3))
    return cv


# ---------------------------------------------------------------- tridiag.f
def test_tridiag_family_bitexact():
    rng = np.random.default_rng(11)
    for NN in (1, 2, 7, 193):
        A = np.asfortranarray(rng.standard_normal((NN, 3)))
        A[:, 1] += 6.0
        B = rng.standard_normal(NN)
        Bc = rng.standard_normal(NN) + 1j * rng.standard_normal(NN)
        A1, B1, A2, B2 = A.copy(order="F"), B.copy(), A.copy(order="F"), B.copy()
        O.tridiag(A1, B1)
        G.tridiag(A2, B2, NN)
        assert bit_equal(A1, A2) and bit_equal(B1, B2)
        A1, C1, A2, C2 = A.copy(order="F"), Bc.copy(), A.copy(order="F"), Bc.copy()
        O.ctridiag(A1, C1)
        G.ctridiag(A2, C2, NN)
        assert bit_equal(A1, A2) and bit_equal(C1, C2)
        M = 5
        BB = np.asfortranarray(rng.standard_normal((M, NN)))
        A1, B1, A2, B2 = A.copy(order="F"), BB.copy(order="F"), A.copy(order="F"), BB.copy(order="F")
        O.trid2(A1, B1)
        G.trid2(A2, B2, M, NN)
        assert bit_equal(A1, A2) and bit_equal(B1, B2)


# -------------------------------------------------------- periodic_implicit.f
def test_tdma_cyclic_bitexact():
    rng = np.random.default_rng(12)
    for n in (1, 5, 64, 498, 700):
        a, b, c, r = (rng.standard_normal(n + 2) for _ in range(4))
        b += 6.0
        u1 = O.tdma(a, b, c, r, n)
        u2 = np.zeros(n + 2)
        G.tdma(a, b, c, r, u2, n)
        assert bit_equal(u1, u2)
        x1 = O.cyclic(a, b, c, -0.7, 0.3, r, n)
        x2 = np.zeros(n + 2)
        G.cyclic(a, b, c, -0.7, 0.3, r, x2, n)
        assert bit_equal(x1, x2)


def test_single_line_solvers_bitexact():
    rng = np.random.default_rng(13)
    n = 37
    g, go = grid(n, n, n)
    Re, Sc, dt, eta = 300.0, 0.71, 0.01, 1.0e4
    cu = rng.random(n)
    cu[cu < 0.5] = 0.0
    s0 = rng.standard_normal(n + 2)
    # implicit_solver (periodic_implicit.f:1)
    a, b = s0.copy(), s0.copy()
    O.implicit_solver(a, n, g["dx"], g["dx12"], Re, dt, 0.0, 0.0, eta, cu)
    G.implicit_solver(b, n, g["dx"], g["dx12"], Re, dt, 0.0, 0.0, eta, cu)
    assert bit_equal(a, b)
    # implicit_uy / implicit_vy
    for fo, fg in ((O.implicit_uy, G.implicit_uy), (O.implicit_vy, G.implicit_vy)):
        a, b = s0.copy(), s0.copy()
        fo(a, n, g["dy"], g["dy12"], Re, dt, 0.25, -0.5, eta, cu)
        fg(b, n, g["dy"], g["dy12"], Re, dt, 0.25, -0.5, eta, cu)
        assert bit_equal(a, b)
    # implicit_Ty / implicit_Tx with non-uniform conductivity and rhoCp
    ll = 0.5 + rng.random(n + 2)
    rr = 0.5 + rng.random(n + 2)
    cu2 = np.concatenate([[0.0], cu, [0.0]])
    a, b = s0.copy(), s0.copy()
    O.implicit_ty(a, n, g["dy"], g["dy12"], Re, Sc, dt, ll, rr, 2.0, 0.0, cu2, eta)
    G.implicit_ty(b, n, g["dy"], g["dy12"], Re, Sc, dt, ll, rr, 2.0, 0.0, cu2, eta)
    assert bit_equal(a[1:n + 1], b[1:n + 1]) and b[0] == s0[0] and b[n + 1] == s0[n + 1]
    a, b = s0.copy(), s0.copy()
    O.implicit_tx(a, n, g["dx"], g["dx12"], Re, Sc, dt, ll, rr, 0.0, 0.0, eta, cu2)
    G.implicit_tx(b, n, g["dx"], g["dx12"], Re, Sc, dt, ll, rr, 0.0, 0.0, eta, cu2)
    assert bit_equal(a, b)


# -------------------------------------------------------------- p2s / s2p
# (256, 3, 256), (256, 2, 48), (32, 3, 256): the register-resident 256-point kernels
@pytest.mark.parametrize("n", [(8, 4, 6), (16, 5, 12), (96, 3, 160), (64, 4, 30),
                               (256, 3, 256), (256, 2, 48), (32, 3, 256)])
def test_p2s_s2p(n):
    nx, ny, nz = n
    rng = np.random.default_rng(14)
    FP = rand_field(rng, nx, ny, nz)
    H = nx // 2 + 1
    sentinel = 7.0 + 3.0j
    F1 = np.full((H, ny + 2, nz + 2), sentinel, order="F")
    F2 = F1.copy(order="F")
    O.p2s(FP, nx, ny, nz, F1)
    G.p2s(FP, F2, nx, ny, nz)
    sl = (slice(None), slice(1, ny + 1), slice(0, nz))
    assert rel_l2(F2[sl], F1[sl]) < 1e-14
    written = np.zeros(F1.shape, bool)
    written[sl] = True
    assert np.all(F2[~written] == sentinel)
    P1 = O.field(nx, ny, nz, -9.0)
    P2 = P1.copy(order="F")
    O.s2p(F1, nx, ny, nz, P1)
    G.s2p(F1, P2, nx, ny, nz)
    box = (slice(0, nx + 1), slice(1, ny + 1), slice(0, nz + 1))
    assert rel_l2(P2[box], P1[box]) < 1e-14
    wr = np.zeros(P1.shape, bool)
    wr[box] = True
    assert np.all(P2[~wr] == -9.0)
    # round trip: s2p(p2s(f)) = f on the sampled cells
    assert rel_l2(P2[0:nx, 1:ny + 1, 0:nz], FP[0:nx, 1:ny + 1, 0:nz]) < 1e-14


# --------------------------------------------------------- SPN / SP0B / PHIBC
def test_spn_sp0b_phibc():
    nx, ny, nz = 16, 12, 10
    g, go = grid(nx, ny, nz)
    rng = np.random.default_rng(15)
    AC, KXZ = O.mkp_coeffs(go)
    H = nx // 2 + 1
    PT = np.asfortranarray(rng.standard_normal((H, ny + 2, nz + 2)) +
                           1j * rng.standard_normal((H, ny + 2, nz + 2)))
    A, B = PT.copy(order="F"), PT.copy(order="F")
    O.spn(nx, ny, nz, AC, KXZ, A)
    G.spn(nx, ny, nz, AC, KXZ, B)
    assert rel_l2(B, A) < 1e-13
    A, B = PT.copy(order="F"), PT.copy(order="F")
    O.sp0b(nx, ny, nz, AC, A)
    G.sp0b(nx, ny, nz, AC, B)
    # the legacy SP0B kernel is built without FMA contraction: exact
    assert bit_equal(A, B)
    PHI = rand_field(rng, nx, ny, nz)
    a, b = PHI.copy(order="F"), PHI.copy(order="F")
    O.phibc(nx, ny, nz, a)
    G.phibc(nx, ny, nz, b)
    assert bit_equal(a, b)


# ---------------------------------------------------------------------- MKP
@pytest.mark.parametrize("n", SIZES)
def test_mkp(n):
    nx, ny, nz = n
    g, go = grid(nx, ny, nz)
    rng = np.random.default_rng(16)
    names = ("p", "u_temp", "v_temp", "w_temp", "u_ta", "v_ta", "w_ta", "u_ep2", "v_ep2",
             "w_ep2", "divu", "u", "v", "w")
    ref = {k: rand_field(rng, nx, ny, nz) for k in names}
    gpu = {k: v.copy(order="F") for k, v in ref.items()}
    dt = 0.013
    O.mkp(go, ref["p"], ref["u_temp"], ref["v_temp"], ref["w_temp"], dt, ref["u_ta"],
          ref["v_ta"], ref["w_ta"], ref["u_ep2"], ref["v_ep2"], ref["w_ep2"], ref["divu"],
          ref["u"], ref["v"], ref["w"])
    G.mkp(gpu["p"], gpu["u_temp"], gpu["v_temp"], gpu["w_temp"], dt, g["dx"], g["dy"], g["dz"],
          g["dx12"], g["dy12"], g["dz12"], 1.0, nx, ny, nz, 1, gpu["u_ta"], gpu["v_ta"],
          gpu["w_ta"], gpu["u_ep2"], gpu["v_ep2"], gpu["w_ep2"], gpu["divu"], gpu["u"],
          gpu["v"], gpu["w"], g["xl"], g["zl"])
    for k in names:
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    # untouched ghost planes stay bit-identical
    for k in ("u", "v", "w", "u_ta"):
        assert bit_equal(gpu[k][nx + 1], ref[k][nx + 1])
        assert bit_equal(gpu[k][:, ny + 1], ref[k][:, ny + 1])


# ------------------------------------------------------------- set_levelset
def test_set_levelset(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    nx, ny, nz = 24, 20, 16
    g, go = grid(nx, ny, nz)
    phi0 = W.sphere_phi0(g, (np.pi, 0.1, np.pi / 2), 0.8)
    phi_ref, cv_ref = O.set_levelset(go, phi0)
    phi = np.zeros_like(phi0)
    cv = np.full((nx, ny, nz, 4), 5.0, order="F")
    G.set_levelset(nx, ny, nz, g["dx"], g["dx12"], g["dy12"], g["dz12"], phi0, phi, g["x"],
                   g["y"], g["z"], cv)
    assert bit_equal(phi, phi_ref)
    assert maxdiff(cv[..., 0], cv_ref[..., 0]) < 4e-16
    assert np.all(cv[..., 1:] == 5.0)
    text = (tmp_path / "cellvalue1.vtk").read_text().splitlines()
    assert text[0] == "# vtk DataFile Version 3.8.1" and text[4] == "DIMENSIONS   24  20  16"
    vals = np.array([float(s) for s in text[-nx * ny * nz:]])
    assert np.allclose(vals, cv_ref[..., 0].ravel(order="F"), atol=1e-7)


# ------------------------------------------------------------- tier-2 step
@pytest.mark.parametrize("n", SIZES)
def test_step_routines_bitexact(n):
    nx, ny, nz = n
    g, go = grid(nx, ny, nz)
    rng = np.random.default_rng(17)
    f = lambda s=1.0: rand_field(rng, nx, ny, nz, s)
    dt, Re, Sc, eta = 0.004, 500.0, 0.71, 1.0e4
    u, v, w, p, T = f(), f(), f(), f(), f()
    # set_bc
    a = [x.copy(order="F") for x in (u, v, w, p, T)]
    b = [x.copy(order="F") for x in (u, v, w, p, T)]
    O.set_bc(*a)
    G.set_bc(b[0], b[1], b[2], b[3], nx, ny, nz, b[4])
    for x, y in zip(a, b):
        assert bit_equal(x, y)
    u, v, w, p, T = a
    # set_convect
    r = [f() for _ in range(3)]
    s = [x.copy(order="F") for x in r]
    O.set_convect(u, r[0], v, r[1], w, r[2], dt, go)
    G.set_convect(u, s[0], v, s[1], w, s[2], dt, nx, ny, nz, g["dx"], g["dy"], g["dz"],
                  g["dx12"], g["dy12"], g["dz12"])
    for x, y in zip(r, s):
        assert bit_equal(x, y)
    # set_convection_for_scalar with a non-uniform rhoCp
    rcp = np.asfortranarray(0.5 + rng.random(u.shape))
    thc = np.asfortranarray(0.5 + rng.random(u.shape))
    r, s = f(), None
    s = r.copy(order="F")
    O.set_convection_for_scalar(u, v, w, dt, go, T, r, rcp)
    G.set_convection_for_scalar(u, v, w, dt, nx, ny, nz, g["dx"], g["dy"], g["dz"], g["dx12"],
                                g["dy12"], g["dz12"], T, s, rcp)
    assert bit_equal(r, s)
    # set_conduction
    r = [f() for _ in range(3)]
    s = [x.copy(order="F") for x in r]
    O.set_conduction(u, r[0], v, r[1], w, r[2], Re, dt, go)
    G.set_conduction(u, s[0], v, s[1], w, s[2], Re, dt, nx, ny, nz, g["dx"], g["dy"], g["dz"],
                     g["dx12"], g["dy12"], g["dz12"])
    for x, y in zip(r, s):
        assert bit_equal(x, y)
    # set_diffusion_for_scalar
    r = f()
    s = r.copy(order="F")
    O.set_diffusion_for_scalar(Re, dt, go, T, r, Sc, thc, rcp)
    G.set_diffusion_for_scalar(Re, dt, nx, ny, nz, g["dx"], g["dy"], g["dz"], g["dx12"],
                               g["dy12"], g["dz12"], T, s, Sc, thc, rcp)
    assert bit_equal(r, s)
    # set_immersed_boundary at l = 1 (builds face masks) and l = 2
    for l in (1, 2):
        cv1 = mask(rng, nx, ny, nz)
        cv2 = cv1.copy(order="F")
        uta, vta, wta = f(), f(), f()
        r = [f() for _ in range(4)]
        s = [x.copy(order="F") for x in r]
        O.set_immersed_boundary(eta, dt, r[0], r[1], r[2], r[3], cv1, uta, vta, wta, l)
        cons = np.array([3.0])
        G.set_immersed_boundary(eta, nx, ny, nz, dt, s[0], s[1], s[2], g["dx"], g["dy"],
                                g["dz"], s[3], cv2, uta, vta, wta, l, cons)
        assert bit_equal(cv1, cv2)
        for x, y in zip(r, s):
            assert bit_equal(x, y)
        assert cons[0] == (0.0 if l == 1 else 3.0)
    # set_explicit / set_explicit_for_tempreture
    for l in (1, 3):
        ins = [f() for _ in range(15)]
        a = [x.copy(order="F") for x in ins]
        b = [x.copy(order="F") for x in ins]
        O.set_explicit(*a, l)
        G.set_explicit(*b, nx, ny, nz, l)
        for x, y in zip(a, b):
            assert bit_equal(x, y)
        ins = [f() for _ in range(5)]
        a = [x.copy(order="F") for x in ins]
        b = [x.copy(order="F") for x in ins]
        O.set_explicit_for_tempreture(*a, l)
        G.set_explicit_for_tempreture(*b, nx, ny, nz, l)
        for x, y in zip(a, b):
            assert bit_equal(x, y)
    # solve_u_temp
    cv = mask(rng, nx, ny, nz)
    ins = [f(0.1) for _ in range(3)]
    a = [x.copy(order="F") for x in ins]
    b = [x.copy(order="F") for x in ins]
    O.solve_u_temp(a[0], a[1], a[2], go, Re, dt, eta, cv, u, v, w)
    G.solve_u_temp(b[0], b[1], b[2], nx, ny, nz, g["dx"], g["dy"], g["dz"], g["dx12"],
                   g["dy12"], g["dz12"], Re, dt, eta, cv, u, v, w)
    for x, y in zip(a, b):
        assert bit_equal(x, y)
    # solve_t with non-uniform rhoCp / thc
    a, b = f(), None
    b = a.copy(order="F")
    O.solve_t(a, go, Re, Sc, dt, rcp, thc, cv, eta)
    G.solve_t(b, nx, ny, nz, g["dx"], g["dy"], g["dz"], g["dx12"], g["dy12"], g["dz12"], Re, Sc,
              dt, rcp, thc, cv, eta)
    assert bit_equal(a, b)


# --------------------------------------------------- parallel_* line drivers
def test_parallel_line_drivers_bitexact():
    """parallel_uy/vy/z/x/Tx/Ty/Tz (nse_dominik.f:2893-3045): each call equals
    the reference's gather, single-line solve (oracle) and scatter on its
    line, bit for bit, and leaves every other entry of the field untouched."""
    rng = np.random.default_rng(29)
    nx, ny, nz = 12, 10, 8
    g, go = grid(nx, ny, nz)
    Re, Sc, dt, eta = 300.0, 0.71, 0.01, 1.0e4
    cv = mask(rng, nx, ny, nz)
    f0 = rand_field(rng, nx, ny, nz)
    rho = np.asfortranarray(0.5 + rng.random(f0.shape))
    thc = np.asfortranarray(0.5 + rng.random(f0.shape))
    d = {"x": (g["dx"], g["dx12"]), "y": (g["dy"], g["dy12"]), "z": (g["dz"], g["dz12"])}

    def vel(name, axis, a, b, ncol, solver, lo, hi_out):
        """gather along `axis` at the other two indices (a, b), 1-based"""
        n = {"x": nx, "y": ny, "z": nz}[axis]
        idx = lambda q: {"x": (q, a, b), "y": (a, q, b), "z": (a, b, q)}[axis]
        cidx = lambda q: {"x": (q - 1, a - 1, b - 1), "y": (a - 1, q - 1, b - 1),
                          "z": (a - 1, b - 1, q - 1)}[axis]
        S = np.zeros(n + 2)
        C = np.zeros(n)
        for q in range(1, hi_in[name] + 1):
            S[q] = f0[idx(q)]
            C[q - 1] = cv[cidx(q) + (ncol - 1,)]
        solver(S, n, *d[axis], Re, dt, 0.0, 0.0, eta, C)
        ref = f0.copy(order="F")
        for q in range(lo, hi_out + 1):
            ref[idx(q)] = S[q]
        got = f0.copy(order="F")
        getattr(G, name)(a, b, got, cv, nx, ny, nz, *d[axis], Re, dt, eta, ncol)
        assert bit_equal(got, ref), name

    hi_in = {"parallel_uy": ny, "parallel_vy": ny - 1, "parallel_z": nz, "parallel_x": nx}
    for (a, b) in ((1, 1), (nx // 2, nz), (nx, 3)):
        vel("parallel_uy", "y", a, b, 2, O.implicit_uy, 0, ny + 1)
        vel("parallel_vy", "y", a, b, 3, O.implicit_vy, 0, ny)
    for (a, b) in ((1, 1), (nx, ny // 2)):
        vel("parallel_z", "z", a, b, 4, O.implicit_solver, 0, nz + 1)
    for (a, b) in ((1, 1), (ny, nz)):
        vel("parallel_x", "x", a, b, 2, O.implicit_solver, 0, nx + 1)

    def temp(name, axis, a, b, solver):
        n = {"x": nx, "y": ny, "z": nz}[axis]
        idx = lambda q: {"x": (q, a, b), "y": (a, q, b), "z": (a, b, q)}[axis]
        S = np.zeros(n + 2)
        R = np.zeros(n + 2)
        L = np.zeros(n + 2)
        C = np.zeros(n + 2)
        for q in range(0, n + 2):
            R[q] = rho[idx(q)]
            L[q] = thc[idx(q)]
            if 1 <= q <= n:
                S[q] = f0[idx(q)]
                i, j, k = idx(q)
                C[q] = cv[i - 1, j - 1, k - 1, 0]
        if axis == "y":
            solver(S, n, *d[axis], Re, Sc, dt, L, R, 0.0, 0.0, C, eta)
        else:
            solver(S, n, *d[axis], Re, Sc, dt, L, R, 0.0, 0.0, eta, C)
        ref = f0.copy(order="F")
        for q in range(1, n + 1):
            ref[idx(q)] = S[q]
        got = f0.copy(order="F")
        # parallel_Tx takes (k, j), parallel_Ty (i, k), parallel_Tz (i, j)
        first, second = (b, a) if axis == "x" else (a, b)
        getattr(G, name)(first, second, nx, ny, nz, rho, thc, got, cv, *d[axis], Re, Sc, dt,
                         eta)
        assert bit_equal(got, ref), name

    temp("parallel_tx", "x", 2, 3, O.implicit_tx)
    temp("parallel_ty", "y", nx, 1, O.implicit_ty)
    temp("parallel_tz", "z", 4, ny, O.implicit_tx)
