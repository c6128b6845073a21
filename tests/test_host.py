"""Host-side logic and the C-ABI surface (no GPU needed)."""
import ctypes
import math
import os
import re
import textwrap

import numpy as np
import pytest

from diablo3_b200 import roofline
from diablo3_b200.grid import create_grid, metrics
from diablo3_b200.params import DbParams, InputError, make_params, read_inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diablo_b200.h")


def test_header_symbols_exported_by_library():
    from diablo3_b200 import lib as L
    lib = L.load()
    src = open(HEADER).read()
    names = set(re.findall(r"^\s*(?:int|const char\*)\s+(db_\w+)\s*\(", src, flags=re.M))
    assert names, "no declarations parsed"
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in the header but not exported"
    assert set(L.EXPORTS) == names
    assert lib.db_abi_version() == 1


def test_params_struct_layout_matches_header():
    # every field of the C struct appears in the ctypes mirror, in order
    src = open(HEADER).read()
    body = src[src.index("typedef struct db_params"):src.index("} db_params;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    cfields = []
    for decl in re.findall(r"(?:int32_t|double)\s+([^;]+);", body):
        for name in decl.split(","):
            cfields.append(re.sub(r"\[.*\]", "", name).strip())
    assert [f for f, _ in DbParams._fields_] == cfields
    assert ctypes.sizeof(DbParams) % 8 == 0


def test_init_without_gpu_fails_cleanly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from diablo3_b200 import lib as L
    p = make_params(nx=32, ny=33, nz=32)
    gy = create_grid(p.ny, lz=2.0, grid_type=1)
    h = ctypes.c_void_p()
    rc = L.load().db_init(ctypes.byref(p), L.dptr(gy), None, ctypes.byref(h))
    assert rc == 2 and not h.value
    assert b"CUDA" in L.load().db_last_error(None)


def test_init_rejects_unsupported_options():
    from diablo3_b200 import lib as L
    gy = create_grid(33, lz=2.0, grid_type=1)
    for bad, code in ((dict(nx=48), 3), (dict(n_th=2), 4), (dict(time_ad_meth=2), 4),
                      (dict(u_bc_ymin=2), 1)):
        p = make_params(nx=32, ny=33, nz=32)
        for k, v in bad.items():
            setattr(p, k, v)
        h = ctypes.c_void_p()
        assert L.load().db_init(ctypes.byref(p), L.dptr(gy), None, ctypes.byref(h)) == code


@pytest.mark.parametrize("gt", [1, 3])
def test_create_grid_walls_and_metrics(gt):
    n = 65
    g = create_grid(n, lz=2.0 if gt == 1 else 1.0, cs=1.5, grid_type=gt)
    assert g.shape == (n + 1,)
    assert np.all(np.diff(g) > 0)
    m = metrics(g)
    lo, hi = (-1.0, 1.0) if gt == 1 else (0.0, 1.0)
    # GF(2) and GF(N+1) are the walls (create_grid.m:60-82)
    assert abs(m["gyf"][1] - lo) < 1e-14 and abs(m["gyf"][n] - hi) < 1e-14
    assert np.allclose(m["dy"][1:], np.diff(m["gyf"]))
    if gt == 1:  # symmetric stretching
        assert np.allclose(g + g[::-1], 0.0, atol=1e-14)


def _write_run(tmp, version="3.4", nth=1):
    (tmp / "grid_def.all").write_text("# Full Grid Resolution\nNx  = 128\nNy  = 96\nNz  = 33\nNth = 1\n")
    (tmp / "input.dat").write_text(textwrap.dedent(f"""\
        C comment
        C comment
        C comment
        C   FLAVOUR       VERSION
            'Front'       {version}
        C   USE_MPI       USE_LES
            .TRUE.        .FALSE.
        C Parameters:     RE      BETA      LX      LY      LZ
                          4.D3    1.0       10.0    2.5     1.5
        C NU_V_SCALE
                          1.5
        C Method:         NUM_PER_DIR       CREATE_NEW_FLOW
                          2                 .TRUE.
        C Time
                  1000           500       0.002     .FALSE.     .TRUE.       0.4      2
        C I/O
                  2               100            1.0              5.0            1.0 0.0 0.5
        C Here include 6*N_TH lines
        C         CREATE_FLOW_TH(1)
                    .TRUE.
        C         FILTER_TH(1)      FILTER_INT(1)
                    .FALSE.           10
        C         RI(1)       PR(1)
                  0.7         2.0
        """))
    (tmp / "input_chan.dat").write_text(textwrap.dedent(f"""\
        C comment
        C comment
        C comment
        C VERSION
           {version}
        C TIME_AD_METH
              1
        C LES:    LES_MODEL_TYPE
                  5
        C ICs:	  IC_TYPE,     KICK,     PHYSICAL_NOISE
                   7           1.D-5      .TRUE.
        C Rotation
                     2.0
        C Aspect Ratio: DELTA
                        3.0
        C Upward vertical vector components, GRAV_X, GRAV_Y, GRAV_Z
                                              0.1     0.2     1.0
        C Forcing:      F_TYPE,   UBULK0,   PX0,    OMEGA0,   AMP_OMEGA0,  FORCE_START
                          2         0.5     0.25     3.0        0.125	    0.5
        C BCs in vertical
        C     u_BC_Zmin,  u_BC_Zmin_C1
              0           0.1
        C     v_BC_Zmin,  v_BC_Zmin_C1
              1           0.2
        C     w_BC_Zmin,  w_BC_Zmin_C1
              0           0.3
        C     u_BC_Zmax,  u_BC_Zmax_C1
              1           0.4
        C     v_BC_Zmax,  v_BC_Zmax_C1
              0           0.5
        C     w_BC_Zmax,  w_BC_Zmax_C1
              1           0.6
        C Here include 6*N_TH lines
        C     TH_BC_Zmin(1),  TH_BC_Zmin_C1(1)
              1               0.7
        C     TH_BC_Zmax(1),  TH_BC_Zmax_C1(1)
              0               0.8
        """))


def test_read_inputs_applies_reference_swaps(tmp_path):
    _write_run(tmp_path)
    p = read_inputs(str(tmp_path))
    # grid_def "Ny"/"Nz" -> code NZ/NY (make_headers:17-21)
    assert (p.nx, p.ny, p.nz) == (128, 33, 96)
    # LX LY LZ read into Lx, Lz, Ly (parameters.f90:101)
    assert (p.lx, p.lz, p.ly) == (10.0, 2.5, 1.5)
    assert p.re == 4000.0 and p.nu_v_scale == 1.5 and p.delta_t == 0.002
    assert p.variable_dt == 1 and p.cfl == 0.4 and p.update_dt == 2
    assert p.ri == 0.7 and p.pr == 2.0 and p.flavor_front == 1
    assert p.ic_type == 7 and p.kick == 1e-5 and p.les_model_type == 5
    assert p.ro == 2.0 and p.delta == 3.0
    # GRAV_X, GRAV_Y, GRAV_Z read into grav_x, grav_z, grav_y (parameters.f90:227)
    assert (p.grav_x, p.grav_z, p.grav_y) == (0.1, 0.2, 1.0)
    assert (p.f_type, p.px0, p.omega0, p.amp_omega0, p.force_start) == (2, 0.25, 3.0, 0.125, 0.5)
    # BC lines in the order u, w, v (parameters.f90:232-242)
    assert (p.u_bc_ymin, p.u_bc_ymin_c1) == (0, 0.1)
    assert (p.w_bc_ymin, p.w_bc_ymin_c1) == (1, 0.2)
    assert (p.v_bc_ymin, p.v_bc_ymin_c1) == (0, 0.3)
    assert (p.u_bc_ymax, p.w_bc_ymax, p.v_bc_ymax) == (1, 0, 1)
    assert (p.th_bc_ymin, p.th_bc_ymin_c1, p.th_bc_ymax, p.th_bc_ymax_c1) == (1, 0.7, 0, 0.8)
    assert p.save_stats_dt == 1.0 and p.save_flow_dt == 100.0


def test_read_inputs_rejects_old_versions(tmp_path):
    _write_run(tmp_path, version="3.3")
    with pytest.raises(InputError):
        read_inputs(str(tmp_path))


def test_reference_setup_parses_when_present():
    """The reference's own finite_front_LES setup files, when the
    DIABLO3_REFERENCE environment variable names a reference checkout."""
    root = os.environ.get("DIABLO3_REFERENCE", "")
    d = os.path.join(root, "setups", "finite_front_LES")
    if not root or not os.path.isdir(d):
        pytest.skip("set DIABLO3_REFERENCE to a reference checkout")
    p = read_inputs(d)
    assert (p.nx, p.ny, p.nz) == (2048, 65, 128)
    assert p.use_les == 1 and p.les_model_type == 5 and p.ic_type == 7


def test_roofline_model_totals():
    # without LES the CN solves run on the spectral state: ~46 P per substep;
    # the reference's sequence (physical solves, transforms of cr and of the
    # new state) ~67 P, ~550 B per point and substep
    p = make_params(nx=512, ny=257, nz=512, variable_dt=1)
    b = roofline.stage_bytes(p)
    u = roofline.units(p)
    total_p = roofline.substep_bytes(p) / u["P"]
    assert 40 < total_p < 50
    assert b["thomas"] == 25 * u["S"] and b["zpass_rhs"] == 8 * u["Xh"] + 8 * u["S"]
    bm = roofline.stage_bytes(make_params(nx=512, ny=257, nz=512, variable_dt=1, precision=1))
    um = roofline.units(make_params(nx=512, ny=257, nz=512, precision=1))
    assert bm["thomas"] == 21 * um["S"] and bm["zpass_rhs"] == 8 * um["Xh"] + 4 * um["S"]
    assert b["inv_x_r"] == b["fwd_x"] == b["fwd_z"] == 0
    ref_p = roofline.reference_substep_bytes(p) / u["P"]
    assert 60 < ref_p < 75
    assert 500 < roofline.reference_substep_bytes(p) / (512 * 257 * 512) < 600
    les = make_params(nx=512, ny=257, nz=512, variable_dt=1, use_les=1)
    assert roofline.stage_bytes(les)["thomas"] == 16 * u["P"]


def test_header_compiles_as_c_and_links(tmp_path):
    """tests/abi_check.c: the header as strict C99, every entry resolved by
    the linker against the built library, error codes without a GPU."""
    import shutil
    import subprocess
    from diablo3_b200 import lib as L
    gcc = shutil.which("gcc")
    if gcc is None or not os.path.exists(L.LIB_PATH):
        pytest.skip("gcc or the built library is missing")
    exe = str(tmp_path / "abi_check")
    libdir = os.path.dirname(L.LIB_PATH)
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "abi_check.c"), "-o", exe, "-L", libdir, "-ldiablo_b200",
                        "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "abi ok" in run.stdout


def test_checkpoint_file_round_trip(tmp_path):
    """checkpoint.save / read on a stand-in channel (no GPU): header,
    parameters (NaN kept), grid, clock and arrays come back unchanged."""
    from diablo3_b200 import checkpoint
    from diablo3_b200 import lib as L

    class Stub:
        def __init__(self):
            self.p = make_params(nx=16, ny=17, nz=16, use_les=1, delta_t=2e-3)
            self.gy = create_grid(17, lz=2.0, grid_type=1)
            rng = np.random.default_rng(0)
            self.state = {f: rng.standard_normal((19, 18, 9)) + 1j * rng.standard_normal((19, 18, 9))
                          for f in L.STATE_FIELDS}
            self.nu = rng.standard_normal((19, 18, 18))

        def status(self):
            s = L.DbStatus()
            s.time, s.time_step, s.delta_t = 1.25, 42, 3e-3
            return s

        def download_state(self):
            return self.state

        def download_field(self, fid):
            return self.nu * (1 if fid == L.NU_T else 2)

    ch = Stub()
    path = str(tmp_path / "x.ckpt")
    checkpoint.save(ch, path)
    hdr, arr = checkpoint.read(path)
    assert hdr["time"] == 1.25 and hdr["time_step"] == 42
    assert hdr["params"]["delta_t"] == 3e-3 and hdr["params"]["dthdx_override"] == "nan"
    assert np.array_equal(np.asarray(hdr["gy"]), ch.gy)
    for f in L.STATE_FIELDS:
        assert np.array_equal(arr[f"spec{f}"], ch.state[f])
    assert np.array_equal(arr["nu_t"], ch.nu) and np.array_equal(arr["kappa_t"], 2 * ch.nu)
    with open(path, "r+b") as fh:
        fh.write(b"NOTMAGIC")
    with pytest.raises(ValueError):
        checkpoint.read(path)


def test_les_filter_weights():
    """les_filter: every LES cell averages the fine cells whose centres it
    holds (weights sum to 1), faces interpolate linearly (exact for a
    linear profile), and a linear mean profile filters to the dyf-weighted
    centres of the LES cells."""
    from diablo3_b200 import les_filter as F
    gf = create_grid(65, lz=2.0, cs=1.5, grid_type=1)
    gc = create_grid(17, lz=2.0, cs=1.5, grid_type=1)
    W, I = F._cell_weights(gf, gc), F._face_interp(gf, gc)
    assert np.allclose(W.sum(axis=1), 1.0) and np.allclose(I.sum(axis=1), 1.0)
    mf, mc = metrics(gf), metrics(gc)
    # every interior fine cell belongs to exactly one interior LES cell
    assert np.allclose(W[1:-1, 1:-1].astype(bool).sum(axis=0), 1.0)
    # faces: linear in y is reproduced exactly
    lin = 3.0 * mf["gy"] - 0.5
    assert np.allclose((I @ lin)[1:], 3.0 * mc["gy"][1:] - 0.5, atol=1e-12)
    # cells: the filtered linear profile is the dyf-weighted mean position of the fine cells
    cen = W @ mf["gyf"]
    for k in range(2, 17):
        assert mc["gy"][k] <= cen[k] <= mc["gy"][k + 1]
    box = F._hbox(np.arange(2 * 8 * 8, dtype=float).reshape(2, 8, 8), 8, 8, 4)
    assert box.shape == (2, 2, 2) and np.isclose(box[0, 0, 0], np.mean([8 * z + x for z in range(4) for x in range(4)]))


def test_profile_error_measures():
    from diablo3_b200 import les_filter as F
    ref0 = {"u1": np.zeros(5)}
    ref = {"u1": np.array([0.0, 1.0, 2.0, 3.0, 0.0])}
    les = {"u1": np.array([0.0, 1.0, 2.0, 2.0, 0.0])}
    rows = slice(1, 4)
    assert np.isclose(F.profile_errors(les, ref, rows)["u1"], 1.0 / np.linalg.norm([1, 2, 3]))
    assert np.isclose(F.evolution_errors(les, ref0, ref, ref0, rows)["u1"], 1.0 / np.linalg.norm([1, 2, 3]))


def test_config3_network_fixture():
    """The DNS-trained closure network the 128x65x128 comparison loads
    (diablo3_b200/closure_study.py made it): parameters, normalisation and
    training range of the 16-64-64-64-2 network, all finite."""
    import numpy as np
    d = np.load(os.path.join(os.path.dirname(__file__), "..", "diablo3_b200", "data", "closure_config3.npz"))
    shapes = {"params": (9538,), "mean": (16,), "std": (16,), "scale": (2,), "lo": (16,), "hi": (16,)}
    for k, sh in shapes.items():
        assert d[k].shape == sh and np.all(np.isfinite(d[k])), k
    assert np.all(d["std"] > 0) and np.all(d["scale"] > 0) and np.all(d["hi"] >= d["lo"])


def test_workloads_and_closure_study_setups():
    """The benchmark configurations and the closure study's DNS / LES
    parameters (no GPU): sizes, closures and the 4x4x4 filter relation."""
    from diablo3_b200 import closure_study
    from diablo3_b200.workloads import WORKLOAD_DESC, workload_params
    c1, c2, c3 = (workload_params(n) for n in ("config1", "config2", "config3"))
    assert (c1.nx, c1.ny, c1.nz, c1.use_les) == (512, 257, 512, 0)
    assert (c2.nx, c2.ny, c2.nz, c2.use_les, c2.les_model_type) == (256, 129, 256, 1, 5)
    assert (c3.nx, c3.ny, c3.nz, c3.ic_type) == (128, 65, 128, 6)
    assert set(WORKLOAD_DESC) >= {"config0", "config1", "slab", "config2", "config3"}
    d = closure_study.dns_params()
    assert (d.nx, d.ny, d.nz, d.use_les, d.variable_dt) == (512, 257, 512, 0, 0)
    a, l = closure_study.les_params(5, 0), closure_study.les_params(6, 1)
    assert (a.nx, a.ny, a.nz) == (d.nx // 4, d.ny // 4 + 1, d.nz // 4) == (l.nx, l.ny, l.nz)
    assert (a.les_model_type, a.precision, l.les_model_type, l.precision) == (5, 0, 6, 1)
    assert a.delta_t == l.delta_t == d.delta_t and a.re == d.re
