"""read_config mirror against the reference's own read_config."""
import pytest

from amrex_euler_allmach_explicit_imex_b200.config import ConfigError, read_config

CASES = [
    {},
    {"amr.n_cell": "400 4", "geometry.prob_hi": "1 0.01", "geometry.is_periodic": "0 1", "euler.problem": "toro1",
     "prob.test": 1, "euler.spatial_order": 2, "euler.cfl": 0.5, "stop_time": 0.2, "max_step": 100000},
    {"euler.problem": "shock_density_bubble_2d"},
    {"problem": "shock_density_bubble", "nx": 2560, "ny": 640},
    {"euler.problem": "gresho_vortex", "euler.vortex_center": "0.5 0.5", "euler.mach": 0.01,
     "euler.pressure": 7142.857142857143, "euler.method": "imex", "euler.spatial_order": 2,
     "euler.imex_acoustic_startup": 0, "euler.imex_picard_iterations": 4, "euler.imex_solver_max_iter": 200},
    {"case": "blob", "order": 2, "riemann": "am_hllc_p", "gamma": 1.67, "cfl": 0.3, "final_time": 0.5,
     "euler.velocity": "0.3 -0.2", "euler.slope_limiter": "van_leer"},
    {"x_lower": -0.5, "x_upper": 0.5, "y_lower": -0.5, "y_upper": 0.5, "euler.field_boundary": "EXACT_DIRICHLET"},
]


@pytest.mark.parametrize("kv", CASES)
def test_matches_reference(ref, kv):
    mine = read_config(kv).cfg.as_dict()
    theirs = ref.configure(kv).as_dict()
    assert mine == theirs


@pytest.mark.parametrize("kv,msg", [
    ({"euler.problem": "shock_density_bubble_2d", "geometry.prob_hi": "4 1"}, "requires domain"),
    ({"euler.method": "imex", "euler.spatial_order": 2}, "acoustic startup off"),
    ({"euler.spatial_order": 3}, "must be 1 or 2"),
    ({"euler.riemann": "roe"}, "Unknown euler.riemann"),
])
def test_rejections_match_reference(ref, kv, msg):
    with pytest.raises(ConfigError, match=msg):
        read_config(kv)
    with pytest.raises(ValueError, match=msg):
        ref.configure(kv)


def test_mach122_variant_accepts_the_imex_method():
    cfg = read_config("euler.problem=shock_bubble_mach122\neuler.method=imex\neuler.spatial_order=2\n"
                      "euler.imex_acoustic_startup=0\n").cfg
    assert cfg.method == 1 and cfg.spatial_order == 2
    assert (cfg.prob_hi[0], cfg.prob_hi[1]) == (4.0, 1.0)
