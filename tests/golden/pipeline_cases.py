"""Scene variants whose distance estimates are pinned against the reference's
own CalculateDistance (oracle/_ref/librefpipe.so, built from the reference's
sources): every formula built here, the Mandelbox rotations, julia mode and
the c constant factor, the DE-function and bailout switches, minN, interior
and iteration-threshold modes, and hybrid sequences with weights, start/stop
iterations, repeat_from, check_for_bailout and the c-constant rule.  Shared
by make_golden.py (which writes the fixture) and tests/test_golden.py.
"""
from mandelbulber2_b200 import abi, configs


def _box(**kw):
    s = configs.mandelbox_scene(kw.pop("scale", -1.5), kw.pop("min_r", 0.5), kw.pop("maxiter", 50))
    return s


def _node(node_type, index=0, level=0, pos=(0.0, 0.0, 0.0), rot=(0.0, 0.0, 0.0), scale=1.0, **kw):
    n = abi.node_defaults(node_type, index, level)
    n.position[:] = list(pos)
    n.rotation[:] = list(rot)
    n.scale = scale
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            getattr(n, k)[:] = list(v)
        else:
            setattr(n, k, v)
    return n


def _tree_scene(slots, prims, nodes, **kw):
    s = abi.scene_defaults(slots[0][0])
    s.n_fractals = len(slots)
    for i, (formula, fkw) in enumerate(slots):
        abi.fractal_defaults(s.fractal[i], formula)
        for k, v in fkw.items():
            setattr(s.fractal[i], k, v)
    s.n_primitives = len(prims)
    for i, (ptype, pkw) in enumerate(prims):
        s.primitive[i] = abi.primitive_defaults(ptype)
        for k, v in pkw.items():
            if isinstance(v, (list, tuple)):
                getattr(s.primitive[i], k)[:] = list(v)
            else:
                setattr(s.primitive[i], k, v)
    s.n_nodes = len(nodes)
    for i, n in enumerate(nodes):
        s.node[i] = n
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _trees():
    F, P = abi.NODE_FRACTAL, abi.NODE_PRIMITIVE
    ADD, MUL, SUB = abi.NODE_BOOLEAN_ADD, abi.NODE_BOOLEAN_MUL, abi.NODE_BOOLEAN_SUB
    box = (abi.FORMULA_MANDELBOX, {"mandelbox_scale": -1.5})
    bulb = (abi.FORMULA_MANDELBULB, {"bulb_power": 8.0})
    menger = (abi.FORMULA_MENGER_SPONGE, {})
    t = {}
    t["tree_two_fractals"] = _tree_scene(
        [box, bulb], [],
        [_node(F, 0, 0, pos=(0.9, 0.0, 0.0), scale=0.5, formula_maxiter=30),
         _node(F, 1, 0, pos=(-0.8, 0.1, 0.0), rot=(10.0, 20.0, 0.0), scale=0.7, formula_maxiter=20)])
    t["tree_intersection"] = _tree_scene(
        [box], [(abi.PRIMITIVE_SPHERE, {"radius": 1.4})],
        [_node(MUL), _node(F, 0, 1, formula_maxiter=30), _node(P, 0, 1)])
    t["tree_subtraction"] = _tree_scene(
        [bulb], [(abi.PRIMITIVE_BOX, {"size": [0.8, 0.8, 3.0], "position": [0.3, 0.0, 0.0], "rotation": [0.0, 0.0, 30.0]})],
        [_node(SUB), _node(F, 0, 1, formula_maxiter=20), _node(P, 0, 1)])
    t["tree_smooth_nested"] = _tree_scene(
        [box, menger], [(abi.PRIMITIVE_TORUS, {"radius": 0.9, "tube_radius": 0.25}),
                        (abi.PRIMITIVE_CYLINDER, {"radius": 0.3, "height": 2.5})],
        [_node(ADD, pos=(0.1, -0.2, 0.05), rot=(5.0, 0.0, 15.0), scale=1.2),
         _node(F, 0, 1, scale=0.6, formula_maxiter=25, julia_mode=1, julia_c=[0.2, -0.1, 0.3]),
         _node(P, 0, 1, smooth_combine=1, smooth_combine_distance=0.3),
         _node(MUL, 0, 1, pos=(0.0, 0.4, 0.0)),
         _node(F, 1, 2, scale=0.8, formula_maxiter=8, fractal_constant_factor=[1.1, 1.0, 0.9]),
         _node(P, 1, 2, rot=(90.0, 0.0, 0.0))])
    t["tree_repeat_detail"] = _tree_scene(
        [bulb], [(abi.PRIMITIVE_PLANE, {"position": [0.0, 0.0, -1.2]})],
        [_node(F, 0, 0, scale=0.3, repeat=[1.0, 1.0, 0.0], detail_level_multiplier=2.0, formula_maxiter=15),
         _node(P, 0, 0)])
    t["tree_disabled_branch"] = _tree_scene(
        [box, bulb], [(abi.PRIMITIVE_SPHERE, {"radius": 0.5}), (abi.PRIMITIVE_SPHERE, {"radius": 0.4, "position": [1.5, 0.0, 0.0]})],
        [_node(ADD), _node(F, 0, 1, formula_maxiter=30), _node(MUL, 0, 1, enabled=0), _node(F, 1, 2),
         _node(P, 0, 2), _node(P, 1, 1)])
    return t


def _pk(maxiter=30, **params):
    s = abi.scene_defaults(abi.FORMULA_PSEUDO_KLEINIAN)
    s.formula_maxiter = maxiter
    for k, v in params.items():
        s.fractal[0].set_param(k, v)
    return s


def _pseudo_kleinian_cases():
    t = {}
    t["pk_default"] = _pk()
    t["pk_params"] = _pk(analyticDE_tweak_005=0.076923, transf_addition_constant_0777=[0.173077, 0.307692, 1.0],
                         transf_minimum_radius_05=0.230769)
    t["pk_sphere_inversion"] = _pk(transf_sphere_inversion_enabled_false=1, transf_stop_iterations_1=2,
                                   transf_offset_000=[0.1, -0.2, 0.3], transf_maxR2_1=1.3,
                                   transf_addition_constantA_000=[0.05, 0.0, -0.1], analyticDE_offset_0=0.2)
    t["pk_prism"] = _pk(transf_function_enabledP_false=1, transf_stop_iterations_P1=3, transf_scale=1.2,
                        transf_constant_multiplier_000=[0.3, 0.2, 0.1])
    t["pk_box_folds"] = _pk(transf_function_enabledBy_false=1, transf_function_enabledBy=0,
                            transf_addition_constant_111=[0.9, 1.1, 1.0], transf_stop_iterations_E=5,
                            transf_function_enabledBx_false=1, transf_scale_1=1.3, transf_start_iterations_A=1)
    s = _pk(transf_function_enabledR_false=1, transf_rotation=[10.0, 20.0, 30.0], transf_start_iterations_R=2,
            transf_addition_constant=[0.1, 0.0, -0.05], transf_function_enabledN_false=1,
            transf_start_iterations_C=1, transf_stop_iterations_C=20)
    s.fractal[0].analytic_de_scale1 = 0.7
    s.fractal[0].mandelbox_folding_limit = 0.9
    t["pk_rotation_flip_scale"] = s
    s = _pk(20)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    s.fractal[0].formula_iterations = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MANDELBOX)
    s.fractal[1].mandelbox_scale = -1.5
    t["hybrid_pk_box"] = s
    s = _pk(25)
    s.delta_de_method = abi.DE_METHOD_FORCE_DELTA
    t["pk_delta"] = s
    return t


def _keyed(formula, maxiter=30, **params):
    s = abi.scene_defaults(formula)
    s.formula_maxiter = maxiter
    for k, v in params.items():
        s.fractal[0].set_param(k, v)
    return s


def _keyed_formula_cases():
    """Box fold bulb pow 2 (16, a delta-DE formula) and Menger mod 1 (61)."""
    t = {}
    t["bfbp2_default"] = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2, 20)
    t["bfbp2_params"] = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2, 20, boxfold_bulbpow2_folding_factor=1.6,
                               boxfold_bulbpow2_z_factor=4.0)
    s = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2, 20, analyticDE_enabled_false=1, analyticDE_offset_2=0.5)
    s.delta_de_method = abi.DE_METHOD_FORCE_ANALYTIC
    s.fractal[0].analytic_de_scale1 = 0.8
    s.fractal[0].analytic_de_offset1 = 0.3
    t["bfbp2_forced_analytic"] = s
    t["menger_mod1_default"] = _keyed(abi.FORMULA_MENGER_MOD1, 12)
    s = _keyed(abi.FORMULA_MENGER_MOD1, 12, transf_constant_multiplier_111=[1.1, 0.9, 1.0],
               transf_rotation_enabled=1, transf_rotation=[5.0, 10.0, -15.0], transf_start_iterations=1,
               transf_scaleD_1=1.1, transf_offset_1=0.5, transf_addition_constant=[0.05, 0.0, -0.02])
    s.fractal[0].transf_scale3 = 2.8
    t["menger_mod1_rotation"] = s
    t["menger_mod1_box_offset_blend"] = _keyed(
        abi.FORMULA_MENGER_MOD1, 12, transf_function_enabledx_false=1, transf_addition_constantA_000=[0.1, 0.2, 0.0],
        transf_function_enabledA_false=1, transf_stop_iterations_A=6, transf_function_enabled_false=1,
        transf_int_A=2, transf_int_B=3, transf_scale_1=0.95, transf_offset=0.1, transf_offset_0=-0.05)
    s = _keyed(abi.FORMULA_MENGER_MOD1, 15)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    s.fractal[0].formula_iterations = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_BOX_FOLD_BULB_POW2)
    t["hybrid_menger_mod1_bfbp2"] = s
    t["bfbp2v2_default"] = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2_V2, 20)
    s = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2_V2, 20, transf_scale=1.2, transf_scale_vary_0=0.1,
               transf_start_iterations_X=1, transf_scaleB_1=0.9, transf_minR2_p25=0.2, transf_maxR2_1=1.1,
               boxfold_bulbpow2_z_factor=4.5, transf_addition_constant_111=[1.0, 0.9, 1.1])
    s.fractal[0].mandelbox_offset[:] = [0.1, 0.0, -0.05]
    s.fractal[0].analytic_de_scale1 = 0.9
    t["bfbp2v2_vary"] = s
    s = _keyed(abi.FORMULA_ABOX_MOD11, 25)
    s.fractal[0].mandelbox_scale = -1.8
    t["abox_mod11_default"] = s
    s = _keyed(abi.FORMULA_ABOX_MOD11, 25, mandelbox_vary_scale_vary=0.1, transf_function_enabled_false=1,
               transf_stop_iterations_D1=4, transf_scale3D_000=[0.3, 0.2, 0.1], transf_function_enabledSw_false=1,
               transf_addition_constant=[0.1, 0.0, 0.05], transf_rotation_enabled=1,
               transf_rotation=[0.0, 15.0, 5.0], transf_stop_iterations_C1=3, transf_scaleG_1=0.97)
    s.fractal[0].mandelbox_scale = 2.2
    s.fractal[0].mandelbox_offset[:] = [0.05, -0.1, 0.0]
    t["abox_mod11_folds"] = s
    s = _keyed(abi.FORMULA_ABOX_MOD11, 25, transf_function_enabledy_false=1, Cpara_para00=0.1, Cpara_paraA=0.3,
               Cpara_paraB=0.2, Cpara_paraC=0.25, Cpara_iterA=3, Cpara_iterB=12, Cpara_iterC=20,
               Cpara_enabledParab_false=1, Cpara_parab_offset0=0.01, Cpara_parab_slope=0.002, Cpara_parab_scale=0.5,
               analyticDE_enabled_false=1, transf_addCpixel_enabled_false=1, transf_alternate_enabled_false=1,
               mandelbulbMulti_order_of_xyz=3, transf_constant_multiplier_111=[0.9, 1.0, 1.1])
    s.fractal[0].mandelbox_scale = -1.7
    s.fractal[0].analytic_de_scale1 = 1.1
    s.fractal[0].analytic_de_offset1 = 0.5
    t["abox_mod11_curve_c"] = s
    s = _keyed(abi.FORMULA_ABOX_MOD11, 20, transf_addCpixel_enabled_false=1, mandelbulbMulti_order_of_xyz=5,
               mandelbox_vary_scale_vary=0.05)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MANDELBULB)
    s.fractal[1].bulb_power = 3.0
    t["hybrid_abox_mod11_bulb"] = s
    t["pkm4_default"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_MOD4, 30)
    t["pkm4_sphere_box"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_MOD4, 30, transf_sphere_inversion_enabled_false=1,
                                  transf_stop_iterations_1=2, transf_offset_000=[0.1, 0.0, -0.1], transf_scaleG_1=1.2,
                                  transf_addition_constantP_000=[0.0, 0.05, 0.0], transf_scaleA_1=0.9,
                                  transf_constant_multiplier_000=[0.1, 0.05, 0.0], transf_start_iterations_M=1)
    t["pkm4_fold_n"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_MOD4, 30, transf_function_enabledG_false=1,
                              transf_addition_constantA_000=[0.05, 0.02, 0.0], transf_function_enabledF_false=1,
                              transf_offsetA_000=[0.9, 1.0, 1.1], transf_function_enabledN_false=1,
                              transf_function_enabledA_false=1, transf_offset_0=0.1, transf_offsetA_0=0.05,
                              transf_function_enabledBx_false=1, transf_function_enabledAx_false=1,
                              transf_offsetA_1=0.8, transf_function_enabledz_false=1)
    t["pksd_default"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_STD_DE, 30)
    t["pksd_benesi"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_STD_DE, 30, transf_benesi_T1_enabled_false=1,
                              transf_stop_iterationsT_1=2, transf_scale3D_222=[2.0, 1.9, 2.1],
                              transf_offset_200=[1.9, 0.1, 0.0], transf_function_enabledx_false=1,
                              transf_start_iterations_D=1, transf_stop_iterationsTM_1=3,
                              transf_function_enabledR_false=1, transf_rotation=[10.0, 0.0, 20.0])
    t["pksd_folds"] = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_STD_DE, 30, transf_function_enabledF_false=1,
                             transf_offsetF_000=[0.5, 0.4, 0.3], transf_offset_000=[0.2, 0.1, 0.0],
                             transf_function_enabledAy=0, transf_function_enabledP_false=1,
                             transf_stop_iterations_P1=2, transf_constant_multiplier_000=[0.2, 0.1, 0.1],
                             transf_stop_iterations_M=2, transf_scaleA_1=0.9, transf_function_enabledAy_false=1,
                             transf_start_iterations_B=3, transf_scaleB_1=1.05, transf_function_enabledN_false=1)
    s = _keyed(abi.FORMULA_PSEUDO_KLEINIAN_STD_DE, 20)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MANDELBOX)
    s.fractal[1].formula_iterations = 2
    s.fractal[1].mandelbox_scale = -1.5
    t["hybrid_pksd_box"] = s
    for gtype in range(8):
        s = _keyed(abi.FORMULA_GENERALIZED_FOLD_BOX, 25, mandelbox_generalized_fold_type=gtype,
                   mandelbox_melt=0.05 * (gtype % 3), mandelbox_solid=1.0 - 0.05 * (gtype % 2))
        s.fractal[0].mandelbox_scale = -1.5 if gtype % 2 else 2.0
        t[f"gfb_type{gtype}"] = s
    s = _keyed(abi.FORMULA_GENERALIZED_FOLD_BOX, 25, mandelbox_generalized_fold_type=5)
    s.fractal[0].mandelbox_main_rotation_enabled = 1
    s.fractal[0].mandelbox_rotation_main[:] = [5.0, -10.0, 20.0]
    s.fractal[0].mandelbox_offset[:] = [0.1, 0.0, 0.0]
    s.fractal[0].mandelbox_folding_min_radius = 0.4
    t["gfb_rotated"] = s
    s = _keyed(abi.FORMULA_MANDELBULB_PUPUKU, 30)
    s.fractal[0].bulb_power = 6.0
    t["pupuku_default"] = s
    s = _keyed(abi.FORMULA_MANDELBULB_PUPUKU, 30, transf_function_enabledP_false=1, transf_function_enabledCx_false=1,
               transf_offsetA_000=[0.1, 0.0, 0.0], transf_function_enabledT_false=1, transf_function_enabledSw_false=1,
               transf_scaleA_1=1.1, transf_function_enabledX_false=1, transf_function_enabledB_false=1,
               transf_scaleB_0=0.3, transf_function_enabledBz_false=1, transf_offset_0=0.2,
               transf_scaleC_1=0.95, analyticDE_enabled_false=1, analyticDE_offset_0=0.1)
    s.fractal[0].bulb_power = 5.0
    s.fractal[0].bulb_alpha_angle_offset = 10.0
    t["pupuku_options"] = s
    s = _keyed(abi.FORMULA_MANDELBULB_PUPUKU, 30, transf_function_enabledC_false=1, transf_function_enabledE_false=1,
               transf_start_iterations_E=2, transf_function_enabledD_false=1)
    s.fractal[0].bulb_power = 4.0
    s.delta_de_function = abi.DE_CUSTOM
    t["pupuku_custom_de"] = s
    t["hextgrid2_default"] = _keyed(abi.FORMULA_DIFS_HEXTGRID2, 20)
    t["hextgrid2_options"] = _keyed(abi.FORMULA_DIFS_HEXTGRID2, 20, transf_function_enabledC_false=1,
                                    transf_stop_iterations_C1=3, transf_offset_2=1.5, transf_function_enabledK_false=1,
                                    transf_scale_vary_0=0.1, transf_function_enabledR_false=1,
                                    transf_rotation=[0.0, 10.0, 30.0], transf_scaleF_1=1.2,
                                    transf_function_enabledJ_false=1, transf_scale_1=0.8)
    t["bfbp2v2_vary_m"] = _keyed(abi.FORMULA_BOX_FOLD_BULB_POW2_V2, 20, transf_scale_vary_0=0.2,
                                 transf_function_enabledM_false=1, transf_stop_iterations_A=8)
    return t


def cases():
    out = {}
    out["bulb_p8"] = configs.mandelbulb_scene(8.0, 250)
    s = configs.mandelbulb_scene(5.0, 60)
    s.fractal[0].bulb_alpha_angle_offset = 12.0
    s.fractal[0].bulb_beta_angle_offset = -7.0
    out["bulb_p5_angles"] = s
    s = configs.mandelbulb_scene(8.0, 40)
    s.julia_mode = 1
    s.julia_c[:] = [0.3, -0.2, 0.1]
    out["bulb_julia"] = s
    s = configs.mandelbulb_scene(8.0, 40)
    s.fractal_constant_factor[:] = [1.2, 1.0, 0.9]
    out["bulb_cmul"] = s
    s = configs.mandelbulb_scene(8.0, 40)
    s.delta_de_function = abi.DE_LINEAR
    out["bulb_linear_de"] = s
    out["box_s-1.5"] = configs.mandelbox_scene(-1.5, 0.5, 50)
    s = configs.mandelbox_scene(2.0, 0.5, 30)
    s.fractal[0].mandelbox_offset[:] = [0.1, -0.2, 0.05]
    out["box_s2_offset"] = s
    s = configs.mandelbox_scene(-1.8, 0.45, 30)
    f = s.fractal[0]
    f.mandelbox_rotations_enabled = 1
    f.mandelbox_rotation_neg[0][:] = [10.0, 0.0, 5.0]
    f.mandelbox_rotation_pos[1][:] = [0.0, -8.0, 0.0]
    f.mandelbox_rotation_pos[2][:] = [3.0, 4.0, -6.0]
    out["box_rotated_folds"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.fractal[0].mandelbox_main_rotation_enabled = 1
    s.fractal[0].mandelbox_rotation_main[:] = [15.0, -10.0, 25.0]
    out["box_main_rotation"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.min_n = 4
    s.use_default_bailout = 0
    s.bailout = 40.0
    s.linear_de_offset = 0.05
    out["box_minn_bailout_offset"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.interior_mode = 1
    out["box_interior"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.iteration_threshold_mode = 1
    out["box_iter_thresh"] = s
    out["menger_12"] = configs.menger_scene(12)
    s = configs.menger_scene(8)
    s.fractal[0].transf_scale3 = 2.6
    s.fractal[0].dont_add_c_constant = 1
    out["menger_s2.6_addc"] = s
    s = abi.scene_defaults(abi.FORMULA_MANDELBULB_POWER2)
    s.formula_maxiter = 40
    out["bulb_power2"] = s
    s = abi.scene_defaults(abi.FORMULA_HYPERCOMPLEX)
    s.formula_maxiter = 40
    out["hypercomplex"] = s
    s = abi.scene_defaults(abi.FORMULA_XENODREAMBUIE)
    s.formula_maxiter = 40
    s.fractal[0].bulb_power = 5.0
    out["xenodreambuie_p5"] = s
    s = abi.scene_defaults(abi.FORMULA_KALEIDOSCOPIC_IFS)
    s.formula_maxiter = 30
    f = s.fractal[0]
    f.ifs_menger_sponge_mode = 1
    f.ifs_scale = 3.0
    f.ifs_rotation_enabled = 1
    f.ifs_rotation[:] = [5.0, 10.0, 0.0]
    out["ifs_menger_mode"] = s
    s = abi.scene_defaults(abi.FORMULA_KALEIDOSCOPIC_IFS)
    s.formula_maxiter = 30
    f = s.fractal[0]
    f.ifs_abs_x = f.ifs_abs_y = f.ifs_abs_z = 1
    for k, d in enumerate(([1.0, 1.0, 0.0], [0.0, 1.0, 1.0], [1.0, 0.0, 1.0])):
        f.ifs_enabled[k] = 1
        f.ifs_direction[k][:] = d
        f.ifs_distance[k] = 0.1 * (k + 1)
        f.ifs_rotations[k][:] = [k * 7.0, 0.0, -k * 3.0]
    out["ifs_vectors"] = s
    out["hybrid_bulb3_menger9"] = configs.hybrid_scene()
    s = configs.hybrid_scene()
    s.fractal[0].formula_weight = 0.6
    s.fractal[1].formula_start_iteration = 2
    s.fractal[1].formula_stop_iteration = 10
    s.formula_maxiter = 20
    out["hybrid_weight_startstop"] = s
    s = abi.scene_defaults(abi.FORMULA_MANDELBOX)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 3
    s.formula_maxiter = 24
    s.fractal[0].mandelbox_scale = -1.6
    s.fractal[0].formula_iterations = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MANDELBULB)
    s.fractal[1].bulb_power = 4.0
    s.fractal[1].check_for_bailout = 0
    abi.fractal_defaults(s.fractal[2], abi.FORMULA_MENGER_SPONGE)
    s.fractal[2].formula_iterations = 3
    s.fractal[2].dont_add_c_constant = 1
    s.repeat_from = 2
    out["hybrid_box_bulb_menger_repeat2"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.limits_enabled = 1
    s.limit_min[:] = [-1.5, -0.8, -2.0]
    s.limit_max[:] = [0.9, 1.2, 0.7]
    out["box_limits"] = s
    s = configs.mandelbulb_scene(8.0, 30)
    s.box_folding = 1
    s.box_folding_limit = 0.9
    s.box_folding_value = 1.7
    out["bulb_global_box_fold"] = s
    s = configs.mandelbulb_scene(6.0, 30)
    s.spherical_folding = 1
    s.spherical_folding_inner = 0.4
    s.spherical_folding_outer = 1.1
    out["bulb_global_spherical_fold"] = s
    s = configs.hybrid_scene()
    s.box_folding = 1
    s.spherical_folding = 1
    s.limits_enabled = 1
    s.limit_min[:] = [-1.0, -1.0, -0.6]
    s.limit_max[:] = [1.0, 0.8, 1.0]
    out["hybrid_folds_limits"] = s
    s = abi.scene_defaults(abi.FORMULA_HYPERCOMPLEX)
    s.formula_maxiter = 30
    s.spherical_folding = 1
    out["hypercomplex_spherical_fold"] = s
    # the delta DE (calculate_distance.cpp:607-760) with each DE function
    for name, base, fn in (("bulb_delta_preferred", configs.mandelbulb_scene(8.0, 30), abi.DE_PREFERRED),
                           ("box_delta_preferred", configs.mandelbox_scene(-1.5, 0.5, 30), abi.DE_PREFERRED),
                           ("box_delta_log", configs.mandelbox_scene(-1.5, 0.5, 30), abi.DE_LOG),
                           ("bulb_delta_pseudo_kleinian", configs.mandelbulb_scene(8.0, 30), abi.DE_PSEUDO_KLEINIAN),
                           ("box_delta_jos_kleinian", configs.mandelbox_scene(-1.5, 0.5, 30), abi.DE_JOS_KLEINIAN),
                           ("menger_delta_custom", configs.menger_scene(10), abi.DE_CUSTOM),
                           ("box_delta_max_axis", configs.mandelbox_scene(2.0, 0.5, 30), abi.DE_MAX_AXIS)):
        base.delta_de_method = abi.DE_METHOD_FORCE_DELTA
        base.delta_de_function = fn
        out[name] = base
    s = configs.hybrid_scene()
    s.delta_de_method = abi.DE_METHOD_FORCE_DELTA
    s.min_n = 3
    out["hybrid_delta"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.delta_de_method = abi.DE_METHOD_FORCE_DELTA
    s.interior_mode = 1
    out["box_delta_interior"] = s
    s = configs.mandelbox_scene(-1.5, 0.5, 30)
    s.delta_de_method = abi.DE_METHOD_FORCE_DELTA
    s.iteration_threshold_mode = 1
    s.limits_enabled = 1
    out["box_delta_iter_thresh_limits"] = s
    # the other analytic DE functions (compute_fractal.cpp:495-621)
    for name, base, fn in (("bulb_pseudo_kleinian", configs.mandelbulb_scene(8.0, 30), abi.DE_PSEUDO_KLEINIAN),
                           ("box_custom", configs.mandelbox_scene(-1.5, 0.5, 30), abi.DE_CUSTOM),
                           ("box_max_axis", configs.mandelbox_scene(-1.5, 0.5, 30), abi.DE_MAX_AXIS)):
        base.delta_de_function = fn
        out[name] = base
    s = configs.hybrid_scene()
    s.delta_de_function = abi.DE_MAX_AXIS
    out["hybrid_max_axis"] = s
    s = configs.hybrid_scene()
    s.delta_de_function = abi.DE_PSEUDO_KLEINIAN
    out["hybrid_pseudo_kleinian"] = s
    # the IFS and a rotated Mandelbox inside hybrids
    s = abi.scene_defaults(abi.FORMULA_MANDELBOX)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 3
    s.formula_maxiter = 30
    s.fractal[0].mandelbox_scale = -1.7
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_KALEIDOSCOPIC_IFS)
    f = s.fractal[1]
    f.ifs_menger_sponge_mode = 1
    f.ifs_scale = 3.0
    f.ifs_rotation_enabled = 1
    f.ifs_rotation[:] = [8.0, 0.0, 4.0]
    abi.fractal_defaults(s.fractal[2], abi.FORMULA_MANDELBULB_POWER2)
    out["hybrid_box_ifs_pow2"] = s
    s = configs.hybrid_scene()
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MANDELBOX)
    s.fractal[1].formula_iterations = 3
    s.fractal[1].mandelbox_scale = -1.6
    s.fractal[1].mandelbox_rotations_enabled = 1
    s.fractal[1].mandelbox_rotation_neg[0][:] = [12.0, 0.0, 3.0]
    s.fractal[1].mandelbox_main_rotation_enabled = 1
    s.fractal[1].mandelbox_rotation_main[:] = [5.0, 9.0, -4.0]
    out["hybrid_bulb_rotated_box"] = s
    # explicit objects trees (calculate_distance.cpp:225-516)
    for name, tree in _trees().items():
        out[name] = tree
    # the pseudo-Kleinian (103), parameters by settings key
    out.update(_pseudo_kleinian_cases())
    out.update(_keyed_formula_cases())
    # quaternion (5) and aexion (19)
    s = abi.scene_defaults(abi.FORMULA_QUATERNION)
    s.formula_maxiter = 40
    out["quaternion"] = s
    s = abi.scene_defaults(abi.FORMULA_AEXION)
    s.formula_maxiter = 40
    out["aexion"] = s
    s = abi.scene_defaults(abi.FORMULA_AEXION)
    s.formula_maxiter = 30
    s.fractal[0].aexion_cadd = -1.1
    s.fractal[0].analytic_de_scale1 = 0.8
    s.fractal[0].analytic_de_offset1 = 0.5
    out["aexion_params"] = s
    s = abi.scene_defaults(abi.FORMULA_AEXION)
    s.formula_maxiter = 30
    s.fractal[0].analytic_de_enabled = 0
    out["aexion_no_analytic_de"] = s
    s = abi.scene_defaults(abi.FORMULA_AEXION)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    s.formula_maxiter = 30
    s.fractal[0].formula_iterations = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_QUATERNION)
    out["hybrid_aexion_quaternion"] = s
    s = abi.scene_defaults(abi.FORMULA_MANDELBULB)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    s.formula_maxiter = 30
    s.fractal[0].bulb_power = 8.0
    s.fractal[0].formula_iterations = 2
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_QUATERNION)
    out["hybrid_bulb_quaternion"] = s
    return out


def render_cases():
    """Small frames rendered by the reference's own render worker (one
    thread, lines in order) with the march jitter drawn from the global
    Park-Miller stream seeded with 1: (name, scene, camera, params).  The
    light is the reference's default main light (its direction is taken from
    the reference and stored with each frame); shading is Lambert with a hard
    or soft, penetrating or not, shadow; AO and specular highlights are off."""
    out = []

    def params(**kw):
        p = configs.base_params(30, kw.pop("vdm", 20.0))
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    sc, cam, p = configs.mandelbulb_512(40, 30, binary_steps=30)
    out.append(("bulb_p8", sc, cam, p))
    sc, cam, p = configs.mandelbox_1080p("A", 48, 27, ao_rays=0)
    p.binary_steps = 30
    out.append(("box_view_a", sc, cam, p))
    out.append(("menger", configs.menger_scene(12), configs.camera((0.0, -3.0, 0.5), width=32, height=32),
                params()))
    out.append(("hybrid_bulb_menger", configs.hybrid_scene(), configs.camera((0.0, -3.0, 0.0), width=40, height=30),
                params()))
    cam = configs.camera((0.15, -1.4, 0.3), fov=360.0, width=48, height=36)
    cam.perspective_type = abi.PROJECTION_EQUIRECTANGULAR
    out.append(("bulb_equirectangular_4x3", configs.mandelbulb_scene(8.0, 20), cam, params()))
    sc, cam, p = configs.mandelbox_1080p("A", 48, 27, ao_rays=0)
    p.binary_steps = 30
    p.advanced_quality = 1
    p.detail_size_max = 0.01
    p.detail_size_min = 0.004
    p.abs_max_marching_step = 0.4
    p.rel_min_marching_step = 0.6
    out.append(("box_advanced_quality", sc, cam, p))
    out.append(("bulb_soft_penetrating", configs.mandelbulb_scene(8.0, 40),
                configs.camera((0.4, -2.4, 0.6), width=32, height=24), params(soft_shadow_cone=10.0, penetrating=1)))
    cases_ = cases()
    out.append(("box_rotated_folds", cases_["box_rotated_folds"], configs.camera((0.0, -5.0, 1.0), width=40, height=24),
                params()))
    cam = configs.camera((0.1, -2.2, 0.4), fov=160.0, width=32, height=32)
    cam.perspective_type = abi.PROJECTION_FISH_EYE
    out.append(("bulb_fish_eye", configs.mandelbulb_scene(8.0, 20), cam, params()))
    cam = configs.camera((0.4, -2.2, 0.9), width=32, height=24)
    cam.legacy_coordinate_system = 1
    out.append(("bulb_legacy_coordinates", configs.mandelbulb_scene(8.0, 20), cam, params()))
    out.append(("box_constant_threshold", configs.mandelbox_scene(-1.5, 0.5, 30),
                configs.camera((0.0, -6.0, 0.0), width=40, height=24), params(constant_de_threshold=1, de_thresh=0.02)))
    s = abi.scene_defaults(abi.FORMULA_KALEIDOSCOPIC_IFS)
    s.formula_maxiter = 30
    f = s.fractal[0]
    f.ifs_scale = 3.0
    f.ifs_offset[:] = [1.0, 1.0, 1.0]
    f.ifs_menger_sponge_mode = 1
    f.ifs_abs_x = f.ifs_abs_y = f.ifs_abs_z = 1
    for k, d in enumerate(([1.0, -1.0, 0.0], [0.0, 1.0, -1.0], [1.0, 0.0, -1.0])):
        f.ifs_enabled[k] = 1
        f.ifs_direction[k][:] = d
    f.ifs_rotation_enabled = 1
    f.ifs_rotation[:] = [20.0, 0.0, 10.0]
    out.append(("ifs_menger", s, configs.camera((1.2, -2.2, 1.5), width=32, height=24), params()))
    out.append(("box_limits_soft_shadow", cases_["box_limits"], configs.camera((0.0, -5.0, 0.5), width=40, height=24),
                params(soft_shadow_cone=15.0)))
    out.append(("bulb_global_folds", cases_["bulb_global_box_fold"],
                configs.camera((0.3, -2.8, 0.4), width=32, height=24), params()))
    out.append(("box_delta_de", cases_["box_delta_preferred"], configs.camera((0.0, -6.0, 0.0), width=40, height=24),
                params()))
    s = abi.scene_defaults(abi.FORMULA_QUATERNION)
    s.formula_maxiter = 30
    out.append(("quaternion", s, configs.camera((0.3, -2.4, 0.8), width=32, height=24), params()))
    out.append(("bulb_slow_shading", configs.mandelbulb_scene(8.0, 20), configs.camera((0.4, -2.2, 0.9), width=24,
                height=16), params(slow_shading=1)))
    out.append(("box_slow_shading", configs.mandelbox_scene(-1.5, 0.5, 20),
                configs.camera((0.0, -6.0, 0.0), width=24, height=16), params(slow_shading=1)))
    sc, cam, p = configs.mandelbulb_512(32, 24, binary_steps=30)
    sc.delta_de_method = abi.DE_METHOD_FORCE_DELTA
    sc.deltade_relative_delta = 0.02
    p.advanced_quality = 1  # the offset is deltade_relative_delta of the detail size
    out.append(("bulb_delta_de_advanced_quality", sc, cam, p))
    s = _pk(60, analyticDE_tweak_005=0.076923, transf_addition_constant_0777=[0.173077, 0.307692, 1.0],
            transf_minimum_radius_05=0.230769)
    cam = configs.camera((2.12066528836305, -3.70836995527439, 1.90220668159675),
                         target=(2.12183734234493, -3.70761659259838, 1.90598160360012), width=32, height=24)
    out.append(("pseudo_kleinian", s, cam, params()))
    trees = _trees()
    out.append(("tree_intersection", trees["tree_intersection"], configs.camera((0.3, -3.5, 1.2), width=32, height=24),
                params()))
    out.append(("tree_smooth_nested", trees["tree_smooth_nested"],
                configs.camera((1.0, -10.0, 2.0), width=32, height=24), params()))
    out.append(("tree_subtraction", trees["tree_subtraction"], configs.camera((0.0, -3.0, 0.3), width=32, height=24),
                params(soft_shadow_cone=15.0)))
    return out
