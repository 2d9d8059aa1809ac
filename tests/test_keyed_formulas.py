"""Formula parameters passed by settings key (mbr_fractal.param): the host
validates each entry against the slot's formula, and the settings reader
fills the list from a [fractal_N] section.  The values and their defaults
are pinned through the reference's own parameter containers: the pipeline
golden vectors of the pseudo-Kleinian cases set the keys by name on the
reference (tests/golden/pipeline_kat.json)."""
import pytest

from mandelbulber2_b200 import abi, settings
from mandelbulber2_b200.render import MbrError, scene_sequence


def _pk():
    return abi.scene_defaults(abi.FORMULA_PSEUDO_KLEINIAN)


def _refused(s, status=abi.MBR_EINVAL):
    with pytest.raises(MbrError) as e:
        scene_sequence(s)
    assert e.value.status == status
    return str(e.value)


def test_known_keys_accepted_and_replaced():
    s = _pk()
    s.fractal[0].set_param("transf_minimum_radius_05", 0.3)
    s.fractal[0].set_param("transf_addition_constant_0777", [0.5, 0.6, 0.9])
    s.fractal[0].set_param("transf_minimum_radius_05", 0.25)
    assert s.fractal[0].n_params == 2
    assert s.fractal[0].params()["transf_minimum_radius_05"][0] == 0.25
    scene_sequence(s)


def test_unknown_key_refused():
    s = _pk()
    s.fractal[0].set_param("transf_scale_3", 2.0)  # a Menger parameter, not read by the pseudo-Kleinian
    _refused(s)


def test_non_finite_value_refused():
    s = _pk()
    s.fractal[0].set_param("transf_addition_constant", [0.0, float("inf"), 0.0])
    _refused(s)


def test_keys_on_a_formula_without_keys_refused():
    s = abi.scene_defaults(abi.FORMULA_MANDELBULB)
    s.fractal[0].set_param("transf_minimum_radius_05", 0.3)
    _refused(s)


def test_param_count_out_of_range_refused():
    s = _pk()
    s.fractal[0].n_params = abi.MBR_MAX_FORMULA_PARAMS + 1
    _refused(s)


def test_unterminated_key_refused():
    import ctypes as C

    s = _pk()
    s.fractal[0].n_params = 1
    C.memmove(C.addressof(s.fractal[0].param[0]), b"x" * abi.MBR_PARAM_KEY_LEN, abi.MBR_PARAM_KEY_LEN)
    _refused(s)


HEADER = "# Mandelbulber settings file\n# version 2.26\n# only modified parameters\n"


def test_settings_reader_fills_the_keys():
    txt = HEADER + ("[main_parameters]\nformula_1 103;\n[fractal_1]\nanalyticDE_tweak_005 0,076923;\n"
                    "transf_addition_constant_0777 0,173077 0,307692 1;\ntransf_minimum_radius_05 0,230769;\n"
                    "transf_function_enabledN_false true;\ntransf_rotation 10 0 -5;\nanalyticDE_scale_1 0,7;\n"
                    "transf_scale_3 2;\n")
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    f = s.scene.fractal[0]
    got = f.params()
    assert got["analyticDE_tweak_005"][0] == 0.076923
    assert got["transf_addition_constant_0777"] == (0.173077, 0.307692, 1.0)
    assert got["transf_minimum_radius_05"][0] == 0.230769
    assert got["transf_function_enabledN_false"][0] == 1.0
    assert got["transf_rotation"] == (10.0, 0.0, -5.0)
    assert "analyticDE_scale_1" not in got and f.analytic_de_scale1 == 0.7  # a named field
    assert "transf_scale_3" not in got  # read into the Menger field, unused here
    scene_sequence(s.scene)
