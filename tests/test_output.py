"""NetCDF output (source/Output.cpp) on CPU: the classic-format writer
against scipy's independent implementation of the format, the reference's
file layout (attributes, dimensions, coordinates, records), and the
oracle's primitive state W against the reference's own build."""
import os
import warnings

import numpy as np
import pytest

from mosscap_b200 import netcdf as nc
from mosscap_b200 import output as out
from mosscap_b200 import problems as P


def _scipy_netcdf():
    warnings.simplefilter("ignore")
    from scipy.io import netcdf_file
    return netcdf_file


@pytest.mark.parametrize("version", [1, 2])
def test_writer_bytes_equal_scipy(tmp_path, version):
    """Same definitions and data, same bytes as scipy.io.netcdf_file."""
    netcdf_file = _scipy_netcdf()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(7)
    q = rng.standard_normal((3, 2, 5, 7))
    dims = [("time", None), ("x", 7), ("y", 5), ("z", 2), ("var", 3)]
    a, b = str(tmp_path / "scipy.nc"), str(tmp_path / "ours.nc")
    f = netcdf_file(a, "w", version=version)
    f.problem = "kh"
    f.num_ghost = np.int32(3)
    f.gamma = np.array([1.4])  # a plain float would be stored as NC_FLOAT by scipy
    for n, s in dims:
        f.createDimension(n, s)
    f.createVariable("x", "d", ("x",))[:] = x
    vt = f.createVariable("time", "d", ("time",))
    vq = f.createVariable("Q", "d", ("time", "var", "z", "y", "x"))
    vt[0], vq[0], vt[1], vq[1] = 0.5, q, 0.7, 2 * q
    f.close()
    w = nc.NcWriter(b, version)
    w.put_att("problem", "kh")
    w.put_att("num_ghost", 3)
    w.put_att("gamma", 1.4)
    for n, s in dims:
        w.create_dim(n, s)
    w.def_var("x", ["x"])
    w.def_var("time", ["time"])
    w.def_var("Q", ["time", "var", "z", "y", "x"])
    w.end_def()
    w.write("x", x)
    w.write_record("time", 0, 0.5)
    w.write_record("Q", 0, q)
    w.write_record("time", 1, 0.7)
    w.write_record("Q", 1, 2 * q)
    w.close()
    assert open(a, "rb").read() == open(b, "rb").read()


@pytest.mark.parametrize("version", [1, 2, 5])
def test_writer_roundtrip_and_append(tmp_path, version):
    """Fixed and record variables, the record dimension defined after the
    others (as the reference does), records added after reopening."""
    path = str(tmp_path / "f.nc")
    rng = np.random.default_rng(1)
    q = [rng.standard_normal((4, 1, 6, 9)) for _ in range(3)]
    w = nc.NcWriter(path, version)
    for n, s in [("x", 9), ("y", 6), ("z", 1), ("time", None), ("var", 4)]:
        w.create_dim(n, s)
    w.put_att("problem", "quad")
    w.put_att("idx", [0, 1, 2])
    w.def_var("x", ["x"])
    w.def_var("time", ["time"])
    w.def_var("Q", ["time", "var", "z", "y", "x"])
    w.end_def()
    w.write("x", np.arange(9.0))
    w.write_record("time", 0, 0.0)
    w.write_record("Q", 0, q[0])
    w.close()
    for r in (1, 2):
        w = nc.NcWriter.append(path)
        assert w.numrecs == r
        w.write_record("time", r, 0.1 * r)
        w.write_record("Q", r, q[r])
        w.close()
    f = nc.read(path)
    assert f.version == version and f.numrecs == 3
    assert f.dims == [("x", 9), ("y", 6), ("z", 1), ("time", None), ("var", 4)]
    assert f.attrs["problem"] == "quad" and list(f.attrs["idx"]) == [0, 1, 2]
    assert np.array_equal(f.variables["time"], [0.0, 0.1, 0.2])
    assert np.array_equal(f.variables["Q"], np.stack(q))
    if version in (1, 2):
        netcdf_file = _scipy_netcdf()
        g = netcdf_file(path, "r", mmap=False)
        assert g.version_byte == version
        assert np.array_equal(g.variables["Q"][:], np.stack(q))
        assert np.array_equal(g.variables["x"][:], np.arange(9.0))
        g.close()


def test_writer_picks_a_version_that_holds_the_file(tmp_path):
    w = nc.NcWriter(str(tmp_path / "a.nc"))
    w.create_dim("n", 10)
    w.def_var("v", ["n"])
    assert w._fits(1)
    big = nc.NcWriter(str(tmp_path / "b.nc"))
    big.create_dim("n", 600 << 20)     # 4.7 GiB of doubles: past the 32-bit variable size
    big.def_var("v", ["n"])
    assert not big._fits(1) and not big._fits(2) and big._fits(5)


class _FakeSim:
    """What write_output reads from a simulation, on the host."""

    def __init__(self, p, seed=0):
        self.problem = p
        self.time = 0.0
        self.rng = np.random.default_rng(seed)
        self._draw()

    def _draw(self):
        self.Q = self.rng.standard_normal(self.problem.shape)
        self.W = self.rng.standard_normal(self.problem.shape)

    def advance(self, t):
        self.time = t
        self._draw()

    def get_Q(self):
        return self.Q

    def get_W(self):
        return self.W

    def eos_fields(self):
        s = self.problem.shape[1:]
        return np.full(s, 0.25), np.full(s, 6000.0)


@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_single_file_layout(tmp_path, ndim):
    """Output.cpp:194-277 with single_file (the default): one file, header
    and axes once, one record of time, Q and W per output."""
    n = {1: (11, 1, 1), 2: (6, 5, 1), 3: (4, 5, 3)}[ndim]
    p = P.Problem("quad", ndim, *n, ng=3, dx=0.1, loc=(-1.0, 2.0, 0.5))
    cfg = out.OutputConfig.for_problem(p, directory=str(tmp_path))
    cfg.variables.primitive = True
    sim = _FakeSim(p)
    recs = []
    for t in (0.0, 0.1, 0.25):
        sim.advance(t)
        out.write_output(sim, cfg)
        recs.append((sim.Q.copy(), sim.W.copy()))
    assert cfg.output_count == 3 and cfg.prev_output_time == 0.25
    f = nc.read(str(tmp_path / "output_quad.nc"))
    nvar, zc, yc, xc = p.shape
    assert f.dims == [("x", xc), ("y", yc), ("z", zc), ("time", None), ("var", nvar)]
    names = ["hydro_program", "hydro_git_hash", "problem", "num_ghost", "single_file", "write_conserved",
             "write_primitive", "write_fluxes", "write_source_term", "irho", "imx", "imy", "imz"][:10 + ndim] + \
        ["iene", "ivx", "ivy", "ivz"][:1 + ndim] + ["ipre"]
    assert list(f.attrs) == names
    assert f.attrs["hydro_program"] == "mosscap" and f.attrs["problem"] == "quad"
    assert int(f.attrs["num_ghost"][0]) == 3 and int(f.attrs["single_file"][0]) == 1
    assert int(f.attrs["iene"][0]) == 1 + ndim and int(f.attrs["ipre"][0]) == 1 + ndim
    assert list(f.var_dims) == ["x", "y", "z"][:ndim] + ["time", "Q", "W"]
    assert f.var_dims["Q"] == ["time", "var", "z", "y", "x"]
    assert np.array_equal(f.variables["time"], [0.0, 0.1, 0.25])
    for r, (q, w) in enumerate(recs):
        assert np.array_equal(f.variables["Q"][r], q)
        assert np.array_equal(f.variables["W"][r], w)
    # State::get_pos: i * dx - (ng - 1/2) dx + loc
    for a, (name, m) in enumerate(zip("xyz", (xc, yc, zc))):
        if a < ndim:
            expect = np.array([k * 0.1 + (-(3 - 0.5) * 0.1) + p.loc[a] for k in range(m)])
            assert np.array_equal(f.variables[name], expect)


def test_file_per_output_and_eos_fields(tmp_path):
    """single_file false: <name>_NNNNN.nc per output with a time dimension
    of one; a non-ideal EOS adds ion_frac and T."""
    p = P.Problem("quad", 2, 6, 5, 1, ng=3, dx=0.1, eos="lte_h_analytic")
    cfg = out.OutputConfig.for_problem(p, name="run", single_file=False, directory=str(tmp_path))
    sim = _FakeSim(p)
    for t in (0.0, 0.5):
        sim.advance(t)
        out.write_output(sim, cfg)
    for k, t in enumerate((0.0, 0.5)):
        f = nc.read(str(tmp_path / f"run_{k:05d}.nc"))
        assert f.numrecs == 0 and ("time", 1) in f.dims
        assert list(f.var_dims) == ["x", "y", "time", "Q", "ion_frac", "T"]
        assert f.var_dims["T"] == ["z", "y", "x"]
        assert np.array_equal(f.variables["time"], [t])
        assert np.all(f.variables["ion_frac"] == 0.25) and np.all(f.variables["T"] == 6000.0)
        assert int(f.attrs["single_file"][0]) == 0 and "ipre" not in f.attrs


def test_flux_and_source_output_refused(tmp_path):
    p = P.Problem("quad", 1, 8, ng=3, dx=0.1)
    cfg = out.OutputConfig.for_problem(p, directory=str(tmp_path))
    cfg.variables.fluxes = True
    with pytest.raises(NotImplementedError):
        out.write_output(_FakeSim(p), cfg)


@pytest.mark.parametrize("case", ["kh_ssprk3", "sod_rk2", "tracers_ssprk4"])
def test_oracle_W_is_the_references(oracle_port, oracle_ref, case):
    """The C restatement's W after a few steps (what the GPU's mc_get_prim
    is compared with) equals the W of the reference's own build bit for bit:
    the primitives of the last stage's input, ghosts included."""
    O = oracle_ref
    if case == "kh_ssprk3":
        p = P.kelvin_helmholtz_2d(32, seed=3)
    elif case == "sod_rk2":
        p = P.sod_1d(256)
    else:
        q = P.random_state(2, 37, 29, ng=3, num_tracers=2, seed=5)
        p = P.Problem("tracers", 2, 37, 29, ng=3, num_tracers=2, dx=1.0 / 37,
                      bc=("periodic", "periodic", "wall", "zerograd", "periodic", "periodic"),
                      reconstruction="muscl", slope_limiter="vanleer", riemann_solver="hllc",
                      time_stepper="ssprk4", gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=1.0, Q=q)
    ws = []
    for kind in ("port", "reference"):
        s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), kind)
        s.set_Q(p.Q)
        s.fill_bcs()
        s.run(3)
        ws.append(s.get_W())
    assert np.array_equal(ws[0].view(np.uint64), ws[1].view(np.uint64))
