"""The case-file readers and writers of include/cosa_io.h, on the CPU:
input.dat parsed into the tables input() builds (src/input.f90:2540-4392,
compared with the table encoding of cosa_b200.tables) and into input()'s
derived values, input.dat / mesh.dat / restart round trips, the gfortran
record framing read back independently in Python (subrecords included), and
the error paths."""
import ctypes as C
import math
import struct

import numpy as np
import pytest

from cosa_b200 import casefiles as cf
from cosa_b200 import cases
from cosa_b200.params import CosaParams, hb_matrix
from cosa_b200.tables import BlockSpec, build_tables

CHANNEL_2BLK = """COSA two-block channel
mesh
n euler internal aircraft
gamma
1.4
time
steady
irest srest cfl lmax iupdt toler (one record split over two lines)
0, 0, 2.5
1000 1 1.d-12
rkap irs
0.3333333333333333 no_irs
ilimf epslimf efx
1 1.0d-6 n
eig_limit_f
n
ilimt epslimt efx
1 1.0d-6 n
eig_limit_t
n
nlevel nl_crs nl_fmg nstart npre npost ncrs
1 99 1 1 1 1 1
preconditioning
none
dgn_cell wri_res wri_tec
n y n
output
bin
forces
none
2
9 5 3 5
1 1 1 1 5 3 21
1 1 1 9 1 3 14
1 5 1 9 5 3 14
1 1 1 9 5 1 80
1 1 3 9 5 3 80
7 5 3 5
7 1 1 7 5 3 91
1 1 1 7 1 3 14
1 5 1 7 5 3 14
1 1 1 7 5 1 80
1 1 3 7 5 3 80
1
1 9 1 1 9 5 3
2 1 1 1 1 5 3 1 2 3
"""

PITCHING_KOM = """COSA k-omega pitching aerofoil
mesh
n komega external aircraft
gamma reyno pranl machfs alpha beta
1.4 6.0d6 0.72 0.3 4.0 0.0
prant tkefar mutfar wall
0.9 1.0d-6 1.0 menter
turcmp lim_prodtke prdlim lim_prodomega fixq order
y n 20.0 n minimum second
time
unsteady hb rkex 2
motion
pitch 0.0127 0.25 0.0 2.5
irest srest cfl cdff lmax iupdt toler
0 0 2.0 1.5 5000 1 1.0d-10
rkap irs
0.3333333333333333 cirs_c 3.0 0
cflt cflit
2.0 3.0
ilimf epslimf efx
1 1.0d-6 y 0.1 1 0.05 n
eig_limit_f
y 0.2 n
ilimt epslimt efx
1 1.0d-6 y 0.1 0 0.05 y
eig_limit_t
n
nlevel nl_crs nl_fmg nstart npre npost ncrs
2 99 1 1 1 1 1
prolongation
bilinear ho_rest lim_corr2 y
preconditioning
none
tref
288.15
dgn_cell wri_res wri_tec
n n n
output
plt
forces
default 0.25 0.0 0.0
lengths
1.0 0.1 1.0
1
2 1 2
2
9 5 2 4
1 1 1 9 1 2 1500
1 5 1 9 5 2 30
1 1 1 9 5 1 80
1 1 2 9 5 2 80
9 5 2 4
1 1 1 9 1 2 1500
1 5 1 9 5 2 30
1 1 1 9 5 1 80
1 1 2 9 5 2 80
2
1 9 1 1 9 5 2
2 1 1 1 1 5 2 1 2 3
2 9 1 1 9 5 2
1 1 1 1 1 5 2 1 2 3
"""


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _tables_equal(a, b):
    for f in ("dims", "nbcs", "bctopo", "cutopo"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


def _face(s, e, t):
    return (tuple(s), tuple(e), t)


def test_channel_tables_match_encoding(tmp_path):
    p, r, t = cf.read_input(_write(tmp_path, "input.dat", CHANNEL_2BLK))
    b1 = BlockSpec(9, 5, 3, [_face((1, 1, 1), (1, 5, 3), 21), _face((1, 1, 1), (9, 1, 3), 14),
                             _face((1, 5, 1), (9, 5, 3), 14), _face((1, 1, 1), (9, 5, 1), 80),
                             _face((1, 1, 3), (9, 5, 3), 80)])
    b2 = BlockSpec(7, 5, 3, [_face((7, 1, 1), (7, 5, 3), 91), _face((1, 1, 1), (7, 1, 3), 14),
                             _face((1, 5, 1), (7, 5, 3), 14), _face((1, 1, 1), (7, 5, 1), 80),
                             _face((1, 1, 3), (7, 5, 3), 80)])
    want = build_tables([b1, b2], [(1, (9, 1, 1), (9, 5, 3), 2, (1, 1, 1), (1, 5, 3), (1, 2, 3))])
    _tables_equal(t, want)
    assert t.ncuts == 2
    # input()'s values: Euler, internal, steady, no IRS -> cfl = vcfl(3)
    assert (p.npde, p.viscous, p.kom, p.harbal, p.moving, p.irsop, p.nlevel) == (5, 0, 0, 0, 0, 0, 1)
    assert p.cfl == 2.5 and p.rat == 1.0 and p.machfs == 0.0 and p.pinf == 1 / 1.4
    assert (r.irest, r.srest, r.lmax, p.iupdt, r.exter, r.wri_res) == (0, 0, 1000, 1, 0, 1)
    assert r.toler == 1e-12 and r.out_format == b"bin" and r.flow_kind == b"aircraft"


def test_pitching_kom_derived_values(tmp_path):
    p, r, t = cf.read_input(_write(tmp_path, "input.dat", PITCHING_KOM))
    assert (p.npde, p.viscous, p.kom, p.harbal, p.nharms, p.moving, p.hbmove) == (7, 1, 1, 1, 2, 1, 1)
    assert p.alpha == 4.0 / 180 * math.pi and p.beta == 0.0
    assert p.reyno == 6.0e6 and p.machfs == 0.3 and p.pranl == 0.72
    tke = 1.0e-6 * 0.3 ** 2
    assert p.tkefar == tke and p.omefar == 1.0 * 1.0 * tke / 1.0 * 6.0e6 / 0.3 and p.mutfar == 1.0
    assert (p.turcmp, p.lim_prodtke, p.lim_prodomega, p.ifixq, p.foturb, p.wallwilc) == (1.0, 0, 0, 1, 0, 0)
    assert p.omegas == 2 * math.pi * 0.0127 and p.omega == p.omegas
    assert p.xh == 0.25 and p.yh == 0.0 and p.dtheta0 == 2.5 / 180.0 * math.pi
    S = 5
    D = np.array(p.dhb[:S * S]).reshape(S, S)
    np.testing.assert_allclose(D, hb_matrix(2, p.omega), rtol=1e-12, atol=1e-14)
    assert r.dt == 2 * math.pi / p.omega / S
    # IRS: cfl = vcfli(3), rat = vcfli(3)/vcfl(3); turbulence likewise
    assert p.irsop == 1 and p.cutcirs == 0 and p.cfl == 3.0 and p.rat == 1.5
    assert p.cflt == 3.0 and p.ratt == 1.5 and p.cdff == 1.5
    # entropy fix: mean-flow type 1; turbulence type 0 plus the mean-flow
    # type (the reference tests etpfxtyp_f for entfx_t_w(2:3))
    assert list(p.entfx_f_w) == [0, 1, 0] and list(p.entfx_t_w) == [1, 1, 0]
    assert p.cntrpy_f == 0.1 and p.entfxctf_f == 0.05 and p.efx_all_f == 0 and p.efx_all_t == 1
    assert p.eig_limit_f == 1 and p.eig_cutoff_f == 0.2 and p.eig_lim_all_f == 0 and p.eig_limit_t == 0
    assert (p.nlevel, p.bln_prol, p.ho_rest, p.lim_corr, p.prd_all_lvls) == (2, 1, 1, 2, 1)
    assert p.stemp == 110.4 / 288.15 and r.tref == 288.15
    assert r.calfor == 1 and list(r.xmom) == [0.25, 0.0, 0.0] and list(r.lngth) == [1.0, 0.1, 1.0]
    assert r.nsurface == 1 and r.n_surblo[0] == 2 and list(r.i_surbl[0][:2]) == [1, 2]
    assert r.out_format == b"plt" and r.exter == 1
    assert t.nblocks == 2 and t.ncuts == 4 and t.bctopo.shape == (8, 10)


def _params_close(a: CosaParams, b: CosaParams):
    for name, typ in CosaParams._fields_:
        va, vb = getattr(a, name), getattr(b, name)
        if hasattr(va, "__len__"):
            va, vb = list(va), list(vb)
        np.testing.assert_allclose(np.asarray(va, dtype=float), np.asarray(vb, dtype=float), rtol=1e-14,
                                   atol=1e-300, err_msg=name)


@pytest.mark.parametrize("text", [CHANNEL_2BLK, PITCHING_KOM], ids=["channel", "pitching_kom"])
def test_input_round_trip(tmp_path, text):
    p, r, t = cf.read_input(_write(tmp_path, "a.dat", text))
    out = str(tmp_path / "b.dat")
    cf.write_input(out, p, r, t)
    p2, r2, t2 = cf.read_input(out)
    _params_close(p2, p)
    _tables_equal(t2, t)
    for f in ("irest", "srest", "lmax", "calfor", "nsurface", "exter", "wri_res"):
        assert getattr(r2, f) == getattr(r, f), f
    assert r2.toler == r.toler and r2.out_format == r.out_format


@pytest.mark.parametrize("make", [
    lambda: cases.partitioned_channel(24, 12, 2, isplit=(10,), jsplit=(5,)),
    lambda: cases.naca0012_ogrid(blocks=(16, 16, 16, 16), nj=8, params=cases.naca_params("kom", nlevel=1)),
    lambda: cases.naca_pitching(nharms=2, blocks=(16, 16), nj=8),
], ids=["partitioned_channel", "naca_kom", "naca_pitching"])
def test_case_tables_round_trip(tmp_path, make):
    """The tables of the library's own cases (permuted blocks, seam cuts)
    written as input.dat and read back unchanged."""
    case = make()
    p = case.params
    if p.kom and p.nlevel > 1:
        p.lim_corr = 1
    r = cf.RunOpts()
    r.lmax, r.toler = 10, 1e-12
    r.exter = 1 if p.aircraft and (p.alpha != 0 or p.harbal) else 0
    r.exter = 1 if (p.viscous or p.harbal) else r.exter
    r.tref = 288.15
    path = str(tmp_path / "input.dat")
    cf.write_input(path, p, r, case.tables)
    p2, r2, t2 = cf.read_input(path)
    _tables_equal(t2, case.tables)
    assert p2.npde == p.npde and p2.harbal == p.harbal and p2.nharms == p.nharms
    assert math.isclose(p2.cfl, p.cfl, rel_tol=1e-14) and math.isclose(p2.rat, p.rat, rel_tol=1e-14)
    if p.harbal:
        S = 2 * p.nharms + 1
        np.testing.assert_allclose(np.array(p2.dhb[:S * S]), np.array(p.dhb[:S * S]), rtol=1e-12, atol=1e-14)
        assert math.isclose(p2.dtheta0, p.dtheta0, rel_tol=1e-14) and p2.hbmove == 1


def _records(path):
    """gfortran sequential records of a file, subrecords joined, with the
    list of (leading, trailing) markers of each piece."""
    data = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(data):
        buf, marks = b"", []
        while True:
            head, = struct.unpack_from("<i", data, pos)
            n = abs(head)
            buf += data[pos + 4:pos + 4 + n]
            tail, = struct.unpack_from("<i", data, pos + 4 + n)
            marks.append((head, tail))
            pos += 8 + n
            if head >= 0:
                break
        out.append((buf, marks))
    return out


def _mesh_case():
    return cases.partitioned_channel(12, 6, 2, isplit=(5,), jsplit=(3,))


def test_mesh_round_trip_and_framing(tmp_path):
    case = _mesh_case()
    t = case.tables
    path = str(tmp_path / "mesh.dat")
    cf.write_mesh(path, t, case.x, case.y, case.z)
    recs = _records(path)
    assert len(recs) == t.nblocks
    for b, ((buf, marks), vx, vy, vz) in enumerate(zip(recs, *(cases.p2_views(t, a) for a in (case.x, case.y, case.z)))):
        im, jm, km = t.dims[b]
        n = im * jm * km
        assert marks == [(24 * n, 24 * n)]
        v = np.frombuffer(buf, "<f8").reshape(3, n)
        for c, w in enumerate((vx, vy, vz)):
            np.testing.assert_array_equal(v[c], w[1:im + 1, 1:jm + 1, 1:km + 1].ravel(order="F"))
    x, y, z = cf.read_mesh(path, t)
    for a, w in zip((x, y, z), (case.x, case.y, case.z)):
        for va, vw in zip(cases.p2_views(t, a), cases.p2_views(t, w)):
            np.testing.assert_array_equal(va[1:-1, 1:-1, 1:-1], vw[1:-1, 1:-1, 1:-1])


def test_mesh_with_displacement_record(tmp_path):
    case = _mesh_case()
    t = case.tables
    _, tot = t.offsets()
    rng = np.random.default_rng(5)
    d = [rng.uniform(0.5, 1.5, tot["p1"]) for _ in range(3)]
    path = str(tmp_path / "mesh.dat")
    cf.write_mesh(path, t, case.x, case.y, case.z, *d)
    recs = _records(path)
    assert len(recs) == 2 * t.nblocks
    out = cf.read_mesh(path, t, with_disp=True)
    for a, w in zip(out[3:], d):
        for va, vw in zip(cases.p1_views(t, a), cases.p1_views(t, w)):
            np.testing.assert_array_equal(va[1:, 1:, 1:, 0], vw[1:, 1:, 1:, 0])
    # a displacement read of a file without the second record fails
    cf.write_mesh(path, t, case.x, case.y, case.z)
    with pytest.raises(cf.CaseFileError):
        cf.read_mesh(path, t, with_disp=True)


def test_mesh_reader_joins_subrecords(tmp_path):
    """A record split into subrecords (negative leading markers on all but
    the last piece, negative trailing markers on all but the first), the
    form gfortran writes above 2 GiB, reads as the one record."""
    case = cases.bump_channel(4, 2, 1)
    t = case.tables
    im, jm, km = t.dims[0]
    n = im * jm * km
    vx, vy, vz = (cases.p2_views(t, a)[0] for a in (case.x, case.y, case.z))
    payload = np.concatenate([w[1:im + 1, 1:jm + 1, 1:km + 1].ravel(order="F") for w in (vx, vy, vz)]).tobytes()
    cuts = [0, 40, 40 + 96, len(payload)]
    blob = b""
    for k in range(3):
        piece = payload[cuts[k]:cuts[k + 1]]
        head = -len(piece) if k < 2 else len(piece)
        tail = len(piece) if k == 0 else -len(piece)
        blob += struct.pack("<i", head) + piece + struct.pack("<i", tail)
    path = tmp_path / "mesh.dat"
    path.write_bytes(blob)
    x, y, z = cf.read_mesh(str(path), t)
    for a, w in zip((x, y, z), (vx, vy, vz)):
        np.testing.assert_array_equal(cases.p2_views(t, a)[0][1:im + 1, 1:jm + 1, 1:km + 1],
                                      w[1:im + 1, 1:jm + 1, 1:km + 1])
    assert len(payload) == 24 * n


def test_restart_round_trip_hb_kom(tmp_path):
    case = _mesh_case()
    t = case.tables
    _, tot = t.offsets()
    npde, nh = 7, 2
    S = 2 * nh + 1
    rng = np.random.default_rng(1)
    q = rng.standard_normal(tot["p3"] * npde * S)
    mut = rng.standard_normal(tot["p3"] * S)
    path = str(tmp_path / "restart")
    cf.write_restart(path, t, npde, q, nharms=nh, mut=mut)
    recs = _records(path)
    assert len(recs) == 2 * t.nblocks
    off, _ = t.offsets()
    for b in range(t.nblocks):
        P3 = int(np.prod(t.dims[b] + 3))
        qb, mb = recs[2 * b][0], recs[2 * b + 1][0]
        np.testing.assert_array_equal(np.frombuffer(qb, "<f8"), q[off["p3"][b] * npde * S:][:P3 * npde * S])
        np.testing.assert_array_equal(np.frombuffer(mb, "<f8"), mut[off["p3"][b] * S:][:P3 * S])
    q2, q1, m2 = cf.read_restart(path, t, npde, nharms=nh, with_mut=True)
    assert q1 is None
    np.testing.assert_array_equal(q2, q)
    np.testing.assert_array_equal(m2, mut)


def test_restart_dual_time_record(tmp_path):
    """q1 at each block's own offset (the reference's writerest hands q1 the
    mut offset, so every block but the first would carry the wrong slice)."""
    case = _mesh_case()
    t = case.tables
    _, tot = t.offsets()
    rng = np.random.default_rng(2)
    q = rng.standard_normal(tot["p3"] * 5)
    q1 = rng.standard_normal(tot["p3"] * 5)
    path = str(tmp_path / "restart")
    cf.write_restart(path, t, 5, q, q1=q1)
    qa, q1a, ma = cf.read_restart(path, t, 5, with_q1=True)
    assert ma is None
    np.testing.assert_array_equal(qa, q)
    np.testing.assert_array_equal(q1a, q1)
    # q1 has no snapshots: harmonic balance with q1 is refused
    with pytest.raises(cf.CaseFileError):
        cf.read_restart(path, t, 5, nharms=1, with_q1=True)


def test_restart_short_file_fails(tmp_path):
    case = _mesh_case()
    t = case.tables
    _, tot = t.offsets()
    path = tmp_path / "restart"
    cf.write_restart(str(path), t, 5, np.zeros(tot["p3"] * 5))
    data = path.read_bytes()
    path.write_bytes(data[:len(data) // 2])
    with pytest.raises(cf.CaseFileError):
        cf.read_restart(str(path), t, 5)
    with pytest.raises(cf.CaseFileError):
        cf.read_restart(str(tmp_path / "missing"), t, 5)
    # a record of the wrong length (npde 7 read as 5)
    cf.write_restart(str(path), t, 7, np.zeros(tot["p3"] * 7))
    with pytest.raises(cf.CaseFileError):
        cf.read_restart(str(path), t, 5)


@pytest.mark.parametrize("edit,code", [
    (lambda s: s.replace("n euler internal", "n spalart internal"), 0x10),
    (lambda s: s.replace("COSA two-block channel\nmesh", "COSA two-block channel\ncgns\ngrid.cgns"), 0x80),
    (lambda s: s.replace("preconditioning\nnone", "preconditioning\nlomach 4 inviscid\nepsp\n1e-5"), 0x10),
    (lambda s: s.replace("1 99 1 1 1 1 1", "4 99 1 1 1 1 1"), 0x10),
    (lambda s: s.replace("output\nbin", "output\nvtk"), 0x10),
    (lambda s: s.replace("1 1.0d-6 n\neig_limit_f", "1 1.0d-6 y 1.5 0 0.1 n\neig_limit_f"), 0x10),
    (lambda s: s[:s.index("7 5 3 5")], 0x10),
], ids=["model", "cgns", "lomach", "nlevel", "format", "cntrpy", "truncated"])
def test_input_errors(tmp_path, edit, code):
    path = _write(tmp_path, "input.dat", edit(CHANNEL_2BLK))
    with pytest.raises(cf.CaseFileError) as e:
        cf.read_input(path)
    assert e.value.code == code


def test_low_speed_preconditioning_lines(tmp_path):
    """The lomach line (cut-off type, viscous/inviscid cut-off) and the
    constant cut-off per level (src/input.f90:3582-3700), read and written
    back; a viscous cut-off in an inviscid run is refused."""
    text = CHANNEL_2BLK.replace("preconditioning\nnone", "preconditioning\nlomach 2 inviscid\nepsp\n2.5d-3")
    p, r, inp = cf.read_input(_write(tmp_path, "input.dat", text))
    assert (p.lomach, p.cutoff_type, p.visprec, p.mixpi, p.uprv) == (1, 2, 0, 0, 0.0)
    assert p.epsp[0] == 2.5e-3
    out = str(tmp_path / "back.dat")
    cf.write_input(out, p, r, inp)
    p2, _, _ = cf.read_input(out)
    assert (p2.lomach, p2.cutoff_type, p2.epsp[0]) == (1, 2, 2.5e-3)
    bad = CHANNEL_2BLK.replace("preconditioning\nnone", "preconditioning\nlomach 2 viscous\nepsp\n1e-5")
    with pytest.raises(cf.CaseFileError):
        cf.read_input(_write(tmp_path, "bad.dat", bad))


def test_default_params_match_python_defaults():
    from cosa_b200.params import default_params
    a, b = cf.default_params(), default_params()
    _params_close(a, b)


# ---- history and force files (src/output.f90:4100-4386, 4941-4965) --------------
def test_hist_record_fortran_e_editing():
    from cosa_b200 import casefiles
    line = casefiles.hist_record(0, 1, [1.234e-3, 2.0, -3.5e-7, 0.0, 1e-120])
    assert line == ("      0        1" + "   0.12340E-02" + "   0.20000E+01" + "  -0.35000E-06" + "   0.00000E+00" +
                    "   0.10000-119\n")
    # rounding to 5 significant digits carries into the exponent
    assert casefiles.hist_record(3, 40, [9.999996]) == "      3       40   0.10000E+02\n"
    # histur.dat: two values end the record after the second field
    assert casefiles.hist_record(0, 10, [1.0, 0.5]) == "      0       10   0.10000E+01   0.50000E+00\n"


def test_force_files_header_and_record():
    from cosa_b200 import casefiles
    from cosa_b200.params import CosaParams
    p = CosaParams()
    names = ',"Cl_p","Cl_v","Cd_p","Cd_v","Cz_p","Cz_v","Cmx_p","Cmx_v","Cmy_p","Cmy_v","Cm_p","Cm_v"'
    assert casefiles.force_header(p) == ' TITLE="Force coefficients"\n VARIABLES="it"' + names + "\n"
    # three surfaces, steady: the reference's list names surface 1's viscous Cm "Cm2_v"
    h3 = casefiles.force_header(p, 3)
    assert h3.count('"Cm2_v"') == 2 and '"Cm1_v"' not in h3
    row = np.arange(12, dtype=float) + 1.0  # gpu.Context.force order
    rec = casefiles.force_record(p, 7, row)
    vals = [row[c] for c in casefiles.FORCE_FILE_COLUMNS]
    body = "".join(" " + ("0.%05dD+%02d" % (round(v * 10 ** (5 - len(str(int(v))))), len(str(int(v))))).rjust(12)
                   for v in vals)
    # i8, then the 12 values on the next record; the exhausted list ends the
    # third record empty (the slash before the second group)
    assert rec == "       7\n" + body + "\n\n"
    # harmonic balance on a pitching grid: 72-column title, time and alpha
    p.harbal, p.moving, p.nharms = 1, 1, 1
    h = casefiles.force_header(p, 1, 2)
    title = h.split("\n")[0]
    assert len(title) == 72 and title.rstrip() == ' TITLE="Force coefficients, Harmonic  2"'
    assert h.split("\n")[1].endswith(',"Cm_v","alpha"')
    h2 = casefiles.force_header(p, 2, 0)
    assert '"Cmy1_v","Cm_p","Cm_v","Cl2_p"' in h2
    rec = casefiles.force_record(p, 5, row, zeit=1.5, alpha_deg=-2.5)
    lines = rec.split("\n")
    assert lines[0] == "       5   0.15000D+01"  # i8, 1x, 1x, d12.5
    assert lines[1] == body and lines[2] == " -0.25000D+01" and lines[3] == ""


def test_output_files_schedule(tmp_path):
    from cosa_b200 import casefiles
    from cosa_b200.params import CosaParams
    p = CosaParams()
    p.npde, p.kom = 7, 1
    out = casefiles.OutputFiles(str(tmp_path), p, iprint=2)
    for it in range(1, 6):
        row = np.full(8, 1.0 / it)
        out.hist(it, row, last=(it == 5))
        out.forces(it, np.ones((1, 12)) * it, last=(it == 5))
    hist = (tmp_path / "hist.dat").read_text().splitlines()
    assert [int(l.split()[1]) for l in hist] == [1, 2, 4, 5]
    assert len((tmp_path / "histur.dat").read_text().splitlines()[0].split()) == 4
    assert (tmp_path / "histg.dat").read_text().splitlines() == [hist[-1]]
    f = (tmp_path / "forces_tec.dat").read_text().split("\n")
    assert f[0] == ' TITLE="Force coefficients"' and f[1].startswith(' VARIABLES="it"')
    assert [int(l) for l in f[2:] if l.strip() and "D" not in l] == [1, 2, 4, 5]
