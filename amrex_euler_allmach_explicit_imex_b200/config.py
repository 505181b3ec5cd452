"""ParmParse-style `key=value` configuration, mirroring the reference's
read_config (amrex/apps/euler_compare/src/euler_compare/core/config_reader.hpp:4-327)
and its selector parsers (core/config_parse_helpers.hpp:3-115).

Input: a dict, a list of "key=value" strings (as on the reference's command
line), or text with one "key = value ..." per line.  Later definitions win,
and a scalar query takes the first token of the last definition, as AMReX
ParmParse does.  Invalid combinations raise ConfigError where the reference
calls amrex::Abort, with the reference's message.

Keys outside the rebuilt hot path (plot files, CSV paths, snapshot settings,
the paper-driver selectors) are accepted and kept in RunSettings.extra.
"""
import dataclasses

from . import abi


class ConfigError(ValueError):
    pass


def _tokens(source):
    """key -> list of tokens (last definition wins)."""
    table = {}
    if source is None:
        return table
    if isinstance(source, dict):
        items = [(k, v) for k, v in source.items()]
        for k, v in items:
            if isinstance(v, (list, tuple)):
                table[k] = [str(x) for x in v]
            else:
                table[k] = str(v).split()
        return table
    lines = source.splitlines() if isinstance(source, str) else list(source)
    for line in lines:
        line = line.split("#", 1)[0]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        k = k.strip()
        if not k or len(k.split()) != 1:
            continue
        table[k] = v.split()
    return table


class _PP:
    def __init__(self, table, prefix=""):
        self.t = table
        self.prefix = prefix

    def _key(self, name):
        return f"{self.prefix}.{name}" if self.prefix else name

    def query(self, name, kind, default):
        v = self.t.get(self._key(name))
        if not v:
            return default, False
        try:
            return kind(v[0]), True
        except ValueError:
            raise ConfigError(f"ParmParse: cannot parse '{v[0]}' for {self._key(name)}")

    def countval(self, name):
        return len(self.t.get(self._key(name), []))

    def queryarr(self, name, kind, default, n):
        v = self.t.get(self._key(name))
        if v is None:
            return list(default)
        out = list(default)
        for i in range(min(n, len(v))):
            out[i] = kind(v[i])
        return out


def _int(s):
    return int(float(s)) if ("e" in s.lower() or "." in s) and float(s).is_integer() else int(s)


def _lower(s):
    return s.lower()


# core/config_parse_helpers.hpp:11-115
def parse_problem(v):
    s = v.lower()
    if s in ("advection_blob", "blob"):
        return abi.PROBLEM["advection_blob"]
    if s in ("toro1", "toro_test_1", "sod", "sod_x"):
        return abi.PROBLEM["toro1"]
    if s in ("gresho", "gresho_vortex"):
        return abi.PROBLEM["gresho_vortex"]
    if s in ("riemann_quadrant", "quadrant_riemann", "liska_wendroff_quadrant"):
        return abi.PROBLEM["riemann_quadrant"]
    if s in ("isentropic_vortex", "bdltv20_isentropic_vortex"):
        return abi.PROBLEM["isentropic_vortex"]
    if s in ("shock_density_bubble_2d", "same_gamma_shock_density_bubble", "shock_density_bubble"):
        return abi.PROBLEM["shock_density_bubble_2d"]
    if s in ("shock_density_bubble_cylindrical_clawpack", "shock_density_bubble_cylindrical",
             "clawpack_shock_density_bubble"):
        return abi.PROBLEM["shock_density_bubble_cylindrical_clawpack"]
    if s in ("shock_bubble_mach122", "shock_density_bubble_mach122"):
        # the [0,4]x[0,1] Mach 1.22 configuration; no ProblemKind in the reference
        return abi.PROBLEM["shock_bubble_mach122"]
    raise ConfigError("Unknown euler.problem=" + v)


def parse_riemann(v):
    s = v.lower()
    if s in ("rusanov", "local_lax_friedrichs", "llf"):
        return abi.RIEMANN["rusanov"]
    if s == "hllc":
        return abi.RIEMANN["hllc"]
    if s in ("lowmach_hllc", "lm_hllc"):
        return abi.RIEMANN["lowmach_hllc"]
    if s in ("xie_am_hllc_p", "am_hllc_p", "xie_hllc_p"):
        return abi.RIEMANN["xie_am_hllc_p"]
    raise ConfigError("Unknown euler.riemann=" + v)


def parse_method(v):
    s = v.lower()
    if s in abi.METHOD:
        return abi.METHOD[s]
    raise ConfigError("Unknown euler.method=" + v)


def parse_imex_form(v):
    if v.lower() in ("bdltv20_t1_s2_source_map_picard", "bdltv20-t1-s2-source-map-picard"):
        return 0
    raise ConfigError("Unknown euler.imex_form=" + v + "; this code pack supports bdltv20_t1_s2_source_map_picard.")


def parse_slope_limiter(v):
    s = v.lower()
    if s == "minmod":
        return abi.LIMITER["minmod"]
    if s in ("mc", "monotonized_central", "monotonized-central"):
        return abi.LIMITER["mc"]
    if s in ("vanleer", "van_leer", "van-leer"):
        return abi.LIMITER["vanleer"]
    raise ConfigError("Unknown euler.slope_limiter=" + v)


def parse_predictor_dissipation(v):
    s = v.lower()
    if s in ("material", "material_speed"):
        return 0
    if s in ("acoustic", "acoustic_speed"):
        return 1
    raise ConfigError("Unknown euler.imex_predictor_dissipation=" + v)


@dataclasses.dataclass
class RunSettings:
    """The parsed configuration: the C-ABI RunConfig plus the string-valued
    settings of RunConfig (core/run_config.hpp:46-54) that the hot path does
    not consume."""

    cfg: abi.RunConfig
    max_grid_size: int = 32
    plot_file: str = "plt"
    plot_int: int = 8
    final_csv: str = ""
    imex_pressure_solver_path: str = "host_single_level_gmres"
    imex_pressure_stabilization: str = "off"
    imex_predictor_dissipation: int = 0
    imex_form: int = 0
    imex_solver_verbose: int = 0
    bdltv20_paper_t1_s2: str = "off"
    extra: dict = dataclasses.field(default_factory=dict)


def default_run_config():
    """RunConfig defaults (core/run_config.hpp:2-55)."""
    c = abi.RunConfig()
    c.n_cell[0], c.n_cell[1] = 64, 64
    c.is_periodic[0], c.is_periodic[1] = 1, 1
    c.prob_lo[0], c.prob_lo[1] = 0.0, 0.0
    c.prob_hi[0], c.prob_hi[1] = 1.0, 1.0
    c.max_step = 8
    c.spatial_order = 1
    c.toro_test = 1
    c.problem = abi.PROBLEM["advection_blob"]
    c.riemann = abi.RIEMANN["hllc"]
    c.method = abi.METHOD["explicit"]
    c.slope_limiter = abi.LIMITER["minmod"]
    c.field_boundary = 0
    c.stop_time = 0.05
    c.gamma = 1.4
    c.cfl = 0.4
    c.imex_cfl = 0.8
    c.imex_acoustic_cfl_cap = 0.0
    c.imex_solver_tol = 1.0e-10
    c.velocity_x, c.velocity_y = 1.0, 0.5
    c.density_inner, c.density_outer = 2.0, 1.0
    c.pressure = 1.0
    c.mach = 0.1
    c.blob_cx, c.blob_cy, c.blob_radius = 0.35, 0.35, 0.15
    c.vortex_cx, c.vortex_cy = 0.0, 0.0
    c.isentropic_vortex_strength = 5.0
    c.riemann_interface_x, c.riemann_interface_y = 0.5, 0.5
    c.imex_solver_max_iter = 100
    c.imex_acoustic_startup = 1
    c.imex_picard_extra_iterations = 1
    c.imex_picard_iterations = 2
    return c


def read_config(source=None):
    """read_config (core/config_reader.hpp:4-327) on key=value input."""
    t = _tokens(source)
    c = default_run_config()
    s = RunSettings(cfg=c)
    pp, amr, geom, eul, prob = _PP(t), _PP(t, "amr"), _PP(t, "geometry"), _PP(t, "euler"), _PP(t, "prob")

    c.max_step, max_step_set = pp.query("max_step", _int, c.max_step)
    c.stop_time, _ = pp.query("stop_time", float, c.stop_time)
    amr_n_cell_set = amr.countval("n_cell") >= 2
    nc = amr.queryarr("n_cell", _int, [c.n_cell[0], c.n_cell[1]], 2)
    c.n_cell[0], c.n_cell[1] = nc
    v, nx_set = pp.query("nx", _int, c.n_cell[0])
    if nx_set:
        c.n_cell[0] = v
    v, ny_set = pp.query("ny", _int, c.n_cell[1])
    if ny_set:
        c.n_cell[1] = v
    grid_size_set = amr_n_cell_set or nx_set or ny_set
    s.max_grid_size, _ = amr.query("max_grid_size", _int, s.max_grid_size)
    s.plot_file, _ = amr.query("plot_file", str, s.plot_file)
    s.plot_int, _ = amr.query("plot_int", _int, s.plot_int)

    lo = geom.queryarr("prob_lo", float, [c.prob_lo[0], c.prob_lo[1]], 2)
    hi = geom.queryarr("prob_hi", float, [c.prob_hi[0], c.prob_hi[1]], 2)
    per = geom.queryarr("is_periodic", _int, [c.is_periodic[0], c.is_periodic[1]], 2)
    c.prob_lo[0], c.prob_lo[1] = lo
    c.prob_hi[0], c.prob_hi[1] = hi
    c.is_periodic[0], c.is_periodic[1] = per
    c.prob_lo[0], _ = pp.query("x_lower", float, c.prob_lo[0])
    c.prob_hi[0], _ = pp.query("x_upper", float, c.prob_hi[0])
    c.prob_lo[1], _ = pp.query("y_lower", float, c.prob_lo[1])
    c.prob_hi[1], _ = pp.query("y_upper", float, c.prob_hi[1])

    c.gamma, _ = eul.query("gamma", float, c.gamma)
    c.cfl, _ = eul.query("cfl", float, c.cfl)
    c.imex_cfl, _ = eul.query("imex_cfl", float, c.imex_cfl)
    c.imex_acoustic_cfl_cap, _ = eul.query("imex_acoustic_cfl_cap", float, c.imex_acoustic_cfl_cap)
    c.imex_solver_tol, _ = eul.query("imex_solver_tol", float, c.imex_solver_tol)
    c.imex_solver_max_iter, _ = eul.query("imex_solver_max_iter", _int, c.imex_solver_max_iter)
    s.imex_solver_verbose, _ = eul.query("imex_solver_verbose", _int, s.imex_solver_verbose)
    c.imex_acoustic_startup, _ = eul.query("imex_acoustic_startup", _int, c.imex_acoustic_startup)
    c.imex_picard_extra_iterations, _ = eul.query("imex_picard_extra_iterations", _int, c.imex_picard_extra_iterations)
    c.imex_picard_iterations, _ = eul.query("imex_picard_iterations", _int, c.imex_picard_iterations)

    problem, _ = eul.query("problem", str, "advection_blob")
    riemann, _ = eul.query("riemann", str, "hllc")
    method, _ = eul.query("method", str, "explicit")
    imex_form, _ = eul.query("imex_form", str, "bdltv20_t1_s2_source_map_picard")
    slope_limiter, _ = eul.query("slope_limiter", str, "minmod")
    dissipation, _ = eul.query("imex_predictor_dissipation", str, "material")
    s.imex_pressure_solver_path, _ = eul.query("imex_pressure_solver_path", str, s.imex_pressure_solver_path)
    field_boundary, _ = eul.query("field_boundary", str, "outflow")
    s.imex_pressure_stabilization, _ = eul.query("imex_pressure_stabilization", str, s.imex_pressure_stabilization)
    s.bdltv20_paper_t1_s2, _ = eul.query("bdltv20_paper_t1_s2", str, s.bdltv20_paper_t1_s2)
    for k in ("bdltv20_paper_pressure_solver", "bdltv20_paper_t1_s2_dt", "bdltv20_paper_epsilon",
              "bdltv20_paper_t1_s2_max_steps", "shock_density_bubble_snapshot_dir",
              "shock_density_bubble_snapshot_times"):
        v, present = eul.query(k, str, None)
        if present:
            s.extra[k] = v
    c.spatial_order, _ = eul.query("spatial_order", _int, c.spatial_order)

    problem, _ = pp.query("case", str, problem)
    problem, _ = pp.query("problem", str, problem)
    method, _ = pp.query("method", str, method)
    riemann, _ = pp.query("riemann", str, riemann)
    c.spatial_order, _ = pp.query("order", _int, c.spatial_order)
    c.spatial_order, _ = pp.query("spatial_order", _int, c.spatial_order)
    c.gamma, _ = pp.query("gamma", float, c.gamma)
    c.cfl, _ = pp.query("cfl", float, c.cfl)
    c.stop_time, _ = pp.query("final_time", float, c.stop_time)

    c.problem = parse_problem(problem)
    c.riemann = parse_riemann(riemann)
    c.method = parse_method(method)
    s.imex_form = parse_imex_form(imex_form)
    c.slope_limiter = parse_slope_limiter(slope_limiter)
    s.imex_predictor_dissipation = parse_predictor_dissipation(dissipation)
    s.bdltv20_paper_t1_s2 = s.bdltv20_paper_t1_s2.lower()
    field_boundary = field_boundary.lower()

    # validation, config_reader.hpp:123-196
    if field_boundary not in ("outflow", "exact_dirichlet"):
        raise ConfigError("euler.field_boundary must be outflow or exact_dirichlet.")
    c.field_boundary = 1 if field_boundary == "exact_dirichlet" else 0
    if c.spatial_order not in (1, 2):
        raise ConfigError("euler.spatial_order must be 1 or 2.")
    if c.imex_picard_extra_iterations < 0:
        raise ConfigError("euler.imex_picard_extra_iterations must be non-negative.")
    if c.imex_picard_iterations < 1:
        raise ConfigError("euler.imex_picard_iterations must be at least one.")
    if c.method == abi.METHOD["imex"]:
        if c.spatial_order != 2:
            raise ConfigError("euler.method=imex requires euler.spatial_order=2 in this code pack.")
        if s.imex_pressure_solver_path != "host_single_level_gmres":
            raise ConfigError("IMEX rows require euler.imex_pressure_solver_path=host_single_level_gmres.")
        if s.imex_pressure_stabilization != "off":
            raise ConfigError("IMEX rows in this code pack use euler.imex_pressure_stabilization=off.")
        if s.imex_predictor_dissipation != 0:
            raise ConfigError("IMEX rows in this code pack use euler.imex_predictor_dissipation=material.")
        if c.slope_limiter != abi.LIMITER["minmod"]:
            raise ConfigError("IMEX rows in this code pack use euler.slope_limiter=minmod.")
        if not (c.imex_acoustic_startup == 0 and c.imex_acoustic_cfl_cap == 0.0):
            raise ConfigError("IMEX rows require material dissipation, acoustic startup off, acoustic cap zero, "
                              "and no pressure stabilization.")

    vel = eul.queryarr("velocity", float, [c.velocity_x, c.velocity_y], 2)
    cen = eul.queryarr("blob_center", float, [c.blob_cx, c.blob_cy], 2)
    vcen = eul.queryarr("vortex_center", float, [c.vortex_cx, c.vortex_cy], 2)
    c.velocity_x, c.velocity_y = vel
    c.blob_cx, c.blob_cy = cen
    c.vortex_cx, c.vortex_cy = vcen
    c.density_inner, _ = eul.query("density_inner", float, c.density_inner)
    c.density_outer, _ = eul.query("density_outer", float, c.density_outer)
    c.pressure, _ = eul.query("pressure", float, c.pressure)
    c.mach, _ = eul.query("mach", float, c.mach)
    c.blob_radius, _ = eul.query("blob_radius", float, c.blob_radius)
    c.isentropic_vortex_strength, _ = eul.query("isentropic_vortex_strength", float, c.isentropic_vortex_strength)
    c.riemann_interface_x, _ = eul.query("riemann_interface_x", float, c.riemann_interface_x)
    c.riemann_interface_y, _ = eul.query("riemann_interface_y", float, c.riemann_interface_y)
    s.final_csv, _ = eul.query("final_csv", str, s.final_csv)
    s.final_csv, _ = pp.query("final_csv", str, s.final_csv)

    c.toro_test, _ = prob.query("test", _int, c.toro_test)
    c.gamma, _ = prob.query("gamma", float, c.gamma)
    c.riemann_interface_x, _ = prob.query("x0", float, c.riemann_interface_x)
    c.riemann_interface_y, _ = prob.query("y0", float, c.riemann_interface_y)

    # shock-density bubble defaults and checks, config_reader.hpp:262-324
    bubble = c.problem in (abi.PROBLEM["shock_density_bubble_2d"],
                           abi.PROBLEM["shock_density_bubble_cylindrical_clawpack"])
    if bubble:
        if not max_step_set and c.max_step == 8:
            c.max_step = 200000
        if not grid_size_set and c.n_cell[0] == 64 and c.n_cell[1] == 64:
            c.n_cell[0], c.n_cell[1] = 160, 40
        if (c.prob_lo[0] == 0.0 and c.prob_lo[1] == 0.0 and c.prob_hi[0] == 1.0 and c.prob_hi[1] == 1.0):
            c.prob_hi[0], c.prob_hi[1] = 2.0, 0.5
        if c.stop_time == 0.05:
            c.stop_time = 0.3
        if c.cfl == 0.4:
            c.cfl = 0.45
        if c.spatial_order == 1:
            c.spatial_order = 2
        c.is_periodic[0], c.is_periodic[1] = 0, 0
        ok = (abs(c.prob_lo[0]) < 1e-14 and abs(c.prob_hi[0] - 2.0) < 1e-14 and abs(c.prob_lo[1]) < 1e-14
              and abs(c.prob_hi[1] - 0.5) < 1e-14)
        if not ok:
            raise ConfigError("shock_density_bubble requires domain x=[0,2], y=[0,0.5].")
        if abs(c.gamma - 1.4) > 1e-14:
            raise ConfigError("shock_density_bubble is a same-gamma ideal-gas test with gamma=1.4.")
        if c.n_cell[0] < 16 or c.n_cell[1] < 4:
            raise ConfigError("shock_density_bubble requires at least 16x4 cells.")
        if not (c.stop_time > 0.0):
            raise ConfigError("shock_density_bubble requires positive finite final_time/stop_time.")
        if not (c.cfl > 0.0):
            raise ConfigError("shock_density_bubble requires positive finite CFL.")
        if c.method == abi.METHOD["explicit"]:
            if c.spatial_order != 2:
                raise ConfigError("shock_density_bubble explicit rows require order/spatial_order=2.")
            if c.riemann not in (abi.RIEMANN["hllc"], abi.RIEMANN["xie_am_hllc_p"]):
                raise ConfigError("shock_density_bubble explicit rows support hllc or xie_am_hllc_p.")
        else:
            if c.problem == abi.PROBLEM["shock_density_bubble_cylindrical_clawpack"]:
                raise ConfigError("cylindrical shock_density_bubble IMEX is not part of the cleaned Cartesian code pack.")
    if c.problem == abi.PROBLEM["shock_bubble_mach122"]:
        # defaults and checks of the Mach 1.22 shock / bubble configuration
        if (c.prob_lo[0] == 0.0 and c.prob_lo[1] == 0.0 and c.prob_hi[0] == 1.0 and c.prob_hi[1] == 1.0):
            c.prob_hi[0], c.prob_hi[1] = 4.0, 1.0
        if c.stop_time == 0.05:
            c.stop_time = 1.0
        if c.cfl == 0.4:
            c.cfl = 0.45
        if c.spatial_order == 1:
            c.spatial_order = 2
        c.is_periodic[0], c.is_periodic[1] = 0, 0
        ok = (abs(c.prob_lo[0]) < 1e-14 and abs(c.prob_hi[0] - 4.0) < 1e-14 and abs(c.prob_lo[1]) < 1e-14
              and abs(c.prob_hi[1] - 1.0) < 1e-14)
        if not ok:
            raise ConfigError("shock_bubble_mach122 requires domain x=[0,4], y=[0,1].")
        if abs(c.gamma - 1.4) > 1e-14:
            raise ConfigError("shock_bubble_mach122 is a same-gamma ideal-gas test with gamma=1.4.")
    return s
