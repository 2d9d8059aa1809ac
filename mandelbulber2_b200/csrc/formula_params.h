// formula_params.h - the formulas whose parameters come by settings key
// (mbr_fractal.param): for each, the keys it reads with the reference's
// defaults (InitFractalParams, src/initparameters.cpp) and the layout of the
// values in a slot's parameter block DevSlot::x.
//
// A value's kind fixes how many x[] entries it takes: an int, a double or a
// bool (0 / 1) one; a vector three; a rotation ten - the zero flag of
// CRotationMatrix and the 3x3 matrix of SetRotation2(angles * pi / 180)
// (src/algebra.cpp:296-302, as sFractal::RecalculateFractalParams builds
// transformCommon.rotationMatrix, src/fractal.cpp:696), row-major.  A NAMED
// entry takes one value from a named mbr_fractal field that holds the same
// parameter (mandelbox_folding_limit, transf_scale3, ...): such keys come
// through those fields, never through mbr_fractal.param.
#pragma once
#include <cmath>

#include "../../include/mbr.h"

#define MBR_SLOT_X 96  // entries of a slot's keyed parameter block

#ifdef __CUDACC__
#define MBR_HD __host__ __device__
#else
#define MBR_HD
#endif

namespace mbr {

enum ParamKind { PK_INT = 0, PK_DOUBLE = 1, PK_BOOL = 2, PK_VEC3 = 3, PK_ROT = 4, PK_NAMED = 5, PK_NAMED3 = 6 };

// the named mbr_fractal fields a NAMED entry reads
enum NamedField {
  NF_MB_LIMIT = 0,   // mandelbox_folding_limit
  NF_MB_VALUE,       // mandelbox_folding_value
  NF_MB_SCALE,       // mandelbox_scale
  NF_ADE_SCALE1,     // analytic_de_scale1 (analyticDE_scale_1)
  NF_ADE_OFFSET1,    // analytic_de_offset1 (analyticDE_offset_1)
  NF_SCALE3,         // transf_scale3 (transf_scale_3)
  NF_MB_OFFSET,      // mandelbox_offset (a vector: NAMED3)
  NF_MB_MIN_R,       // mandelbox_folding_min_radius
  NF_MB_FIXED_R,     // mandelbox_folding_fixed_radius
  NF_POWER,          // bulb_power (power)
  NF_ALPHA,          // bulb_alpha_angle_offset, in radians (fractal.cpp:677)
  NF_BETA            // bulb_beta_angle_offset, in radians (fractal.cpp:678)
};

// formulas that carry orbit state (AuxX) or end orbits by the convergence
// bailout: the FP32 wavefront's iteration does not carry them
inline MBR_HD bool keyed_formula_has_state(int formula) {
  return formula == MBR_FORMULA_PSEUDO_KLEINIAN || formula == MBR_FORMULA_BOX_FOLD_BULB_POW2_V2 ||
         formula == MBR_FORMULA_ABOX_MOD11 || formula == MBR_FORMULA_PSEUDO_KLEINIAN_MOD4 ||
         formula == MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE || formula == MBR_FORMULA_MANDELBULB_PUPUKU ||
         formula == MBR_FORMULA_DIFS_HEXTGRID2;
}

// cFractalPseudoKleinian (formula/definition/fractal_pseudo_kleinian.cpp:
// 30-202): sphere inversion, prism shape, abs-box and box folds, the
// Kleinian fold, rotation and offset.  The box fold reads the slot's
// mandelbox_folding_limit / _value and the Kleinian fold its
// analytic_de_scale1 (mbr_fractal fields, after the keyed block).
enum PseudoKleinianX {
  PKX_SPH_INV = 0,                  // transf_sphere_inversion_enabled_false
  PKX_START_X = 1,                  // transf_start_iterations_X
  PKX_STOP_1 = 2,                   // transf_stop_iterations_1
  PKX_OFFSET000 = 3,                // transf_offset_000 (3)
  PKX_MAXR2 = 6,                    // transf_maxR2_1
  PKX_ADD_A000 = 7,                 // transf_addition_constantA_000 (3)
  PKX_DE_OFFSET0 = 10,              // analyticDE_offset_0
  PKX_PRISM = 11,                   // transf_function_enabledP_false
  PKX_START_P = 12,                 // transf_start_iterations_P
  PKX_STOP_P1 = 13,                 // transf_stop_iterations_P1
  PKX_SCALE = 14,                   // transf_scale
  PKX_CMUL000 = 15,                 // transf_constant_multiplier_000 (3)
  PKX_ABS_BOX = 18,                 // transf_function_enabledBy_false
  PKX_START_E = 19,                 // transf_start_iterations_E
  PKX_STOP_E = 20,                  // transf_stop_iterations_E
  PKX_ADD111 = 21,                  // transf_addition_constant_111 (3)
  PKX_ABS_BOX_Z = 24,               // transf_function_enabledBy
  PKX_BOX = 25,                     // transf_function_enabledBx_false
  PKX_START_A = 26,                 // transf_start_iterations_A
  PKX_STOP_A = 27,                  // transf_stop_iterations_A
  PKX_SCALE1 = 28,                  // transf_scale_1
  PKX_CSIZE = 29,                   // transf_addition_constant_0777 (3)
  PKX_START_C = 32,                 // transf_start_iterations_C
  PKX_STOP_C = 33,                  // transf_stop_iterations_C
  PKX_MINR05 = 34,                  // transf_minimum_radius_05
  PKX_FLIP_Z = 35,                  // transf_function_enabledN_false
  PKX_FLIP_W = 36,                  // transf_function_enabledw_false
  PKX_TWEAK005 = 37,                // analyticDE_tweak_005
  PKX_ROT_ON = 38,                  // transf_function_enabledR_false
  PKX_START_R = 39,                 // transf_start_iterations_R
  PKX_STOP_R = 40,                  // transf_stop_iterations_R
  PKX_ROT = 41,                     // transf_rotation (10)
  PKX_ADD000 = 51,                  // transf_addition_constant (3)
  PKX_MB_LIMIT = 54,                // mandelbox_folding_limit (named)
  PKX_MB_VALUE = 55,                // mandelbox_folding_value (named)
  PKX_DE_SCALE1 = 56,               // analyticDE_scale_1 (named)
  PKX_COUNT = 57
};
static_assert(PKX_COUNT <= MBR_SLOT_X, "pseudo-Kleinian block exceeds the slot's parameter block");

// cFractalBoxFoldBulbPow2 (formula/definition/fractal_box_fold_bulb_pow2.cpp:27-76)
enum BoxFoldBulbPow2X {
  BFX_FOLD = 0,      // boxfold_bulbpow2_folding_factor
  BFX_ZFACTOR = 1,   // boxfold_bulbpow2_z_factor
  BFX_ADE_ON = 2,    // analyticDE_enabled_false
  BFX_ADE_OFFSET2 = 3,  // analyticDE_offset_2
  BFX_ADE_SCALE1 = 4,   // analyticDE_scale_1 (named)
  BFX_ADE_OFFSET1 = 5,  // analyticDE_offset_1 (named)
  BFX_COUNT = 6
};

// cFractalMengerMod1 (formula/definition/fractal_menger_mod1.cpp:29-103)
enum MengerMod1X {
  MMX_CM111 = 0,     // transf_constant_multiplier_111 (3)
  MMX_ROT_ON = 3,    // transf_rotation_enabled
  MMX_START = 4,     // transf_start_iterations
  MMX_STOP = 5,      // transf_stop_iterations
  MMX_ROT = 6,       // transf_rotation (10)
  MMX_SCALED1 = 16,  // transf_scaleD_1
  MMX_OFFSET1 = 17,  // transf_offset_1
  MMX_ADD000 = 18,   // transf_addition_constant (3)
  MMX_BOX_OFF = 21,  // transf_function_enabledx_false
  MMX_START_A = 22,  // transf_start_iterations_A
  MMX_STOP_A = 23,   // transf_stop_iterations_A
  MMX_ADD_A000 = 24, // transf_addition_constantA_000 (3)
  MMX_AVG_SCALE = 27,  // transf_function_enabledA_false
  MMX_BLEND = 28,    // transf_function_enabled_false
  MMX_INT_A = 29,    // transf_int_A
  MMX_INT_B = 30,    // transf_int_B
  MMX_SCALE1 = 31,   // transf_scale_1
  MMX_OFFSET = 32,   // transf_offset
  MMX_OFFSET0 = 33,  // transf_offset_0
  MMX_SCALE3 = 34,   // transf_scale_3 (named)
  MMX_COUNT = 35
};

// cFractalBoxFoldBulbPow2V2 (formula/definition/fractal_box_fold_bulb_pow2_v2.cpp:29-146)
enum BoxFoldBulbPow2V2X {
  B2X_ADD111 = 0,     // transf_addition_constant_111 (3)
  B2X_START_B = 3,    // transf_start_iterations_B
  B2X_STOP_B = 4,     // transf_stop_iterations_B
  B2X_START_S = 5,    // transf_start_iterations_S
  B2X_STOP_S = 6,     // transf_stop_iterations_S
  B2X_MINR2 = 7,      // transf_minR2_p25
  B2X_MAXR2 = 8,      // transf_maxR2_1
  B2X_START_C = 9,    // transf_start_iterations_C
  B2X_STOP_C = 10,    // transf_stop_iterations_C
  B2X_SCALE = 11,     // transf_scale
  B2X_START_X = 12,   // transf_start_iterations_X
  B2X_STOP_X = 13,    // transf_stop_iterations_X
  B2X_SCALE_VARY = 14,  // transf_scale_vary_0
  B2X_SCALE_B1 = 15,  // transf_scaleB_1
  B2X_VARY_M = 16,    // transf_function_enabledM_false
  B2X_START_A = 17,   // transf_start_iterations_A
  B2X_STOP_A = 18,    // transf_stop_iterations_A
  B2X_ZFACTOR = 19,   // boxfold_bulbpow2_z_factor
  B2X_ADE_OFFSET2 = 20,  // analyticDE_offset_2
  B2X_MB_OFFSET = 21,    // mandelbox_offset (named, 3)
  B2X_ADE_SCALE1 = 24,   // analyticDE_scale_1 (named)
  B2X_ADE_OFFSET1 = 25,  // analyticDE_offset_1 (named)
  B2X_COUNT = 26
};

// cFractalAboxMod11 (formula/definition/fractal_abox_mod11.cpp:34-250)
enum AboxMod11X {
  ABX_SCALE_VARY = 0,   // mandelbox_vary_scale_vary
  ABX_ADD111 = 1,       // transf_addition_constant_111 (3)
  ABX_START_B = 4,      // transf_start_iterations_B
  ABX_STOP_B = 5,       // transf_stop_iterations_B
  ABX_FOLD_Z = 6,       // transf_function_enabled
  ABX_FOLD_D = 7,       // transf_function_enabled_false
  ABX_START_D = 8,      // transf_start_iterations_D
  ABX_STOP_D1 = 9,      // transf_stop_iterations_D1
  ABX_SCALE3D = 10,     // transf_scale3D_000 (3)
  ABX_SWAP = 13,        // transf_function_enabledSw_false
  ABX_START_S = 14,     // transf_start_iterations_S
  ABX_STOP_S = 15,      // transf_stop_iterations_S
  ABX_PARA = 16,        // transf_function_enabledy_false
  ABX_CP_LINEAR = 17,   // Cpara_enabledLinear
  ABX_CP_PARA00 = 18,   // Cpara_para00
  ABX_CP_PARAA = 19,    // Cpara_paraA
  ABX_CP_PARAB = 20,    // Cpara_paraB
  ABX_CP_PARAC = 21,    // Cpara_paraC
  ABX_CP_ITERA = 22,    // Cpara_iterA
  ABX_CP_ITERB = 23,    // Cpara_iterB
  ABX_CP_ITERC = 24,    // Cpara_iterC
  ABX_CP_CURVES = 25,   // Cpara_enabledCurves
  ABX_CP_PARAB_ON = 26, // Cpara_enabledParab_false
  ABX_CP_OFFSET0 = 27,  // Cpara_parab_offset0
  ABX_CP_SLOPE = 28,    // Cpara_parab_slope
  ABX_CP_SCALE = 29,    // Cpara_parab_scale
  ABX_MINR2 = 30,       // transf_minR2_p25
  ABX_MAXR2 = 31,       // transf_maxR2_1
  ABX_START_A = 32,     // transf_start_iterations_A
  ABX_STOP_A = 33,      // transf_stop_iterations_A
  ABX_ADE_ON = 34,      // analyticDE_enabled_false
  ABX_ADD000 = 35,      // transf_addition_constant (3)
  ABX_ADDC = 38,        // transf_addCpixel_enabled_false
  ABX_START_E = 39,     // transf_start_iterations_E
  ABX_STOP_E = 40,      // transf_stop_iterations_E
  ABX_ALTERNATE = 41,   // transf_alternate_enabled_false
  ABX_ORDER = 42,       // mandelbulbMulti_order_of_xyz
  ABX_CM111 = 43,       // transf_constant_multiplier_111 (3)
  ABX_ROT_ON = 46,      // transf_rotation_enabled
  ABX_START_R = 47,     // transf_start_iterations_R
  ABX_STOP_R = 48,      // transf_stop_iterations_R
  ABX_ROT = 49,         // transf_rotation (10)
  ABX_START_C = 59,     // transf_start_iterations_C
  ABX_STOP_C1 = 60,     // transf_stop_iterations_C1
  ABX_SCALE_G1 = 61,    // transf_scaleG_1
  ABX_MB_OFFSET = 62,   // mandelbox_offset (named, 3)
  ABX_MB_SCALE = 65,    // mandelbox_scale (named)
  ABX_ADE_SCALE1 = 66,  // analyticDE_scale_1 (named)
  ABX_ADE_OFFSET1 = 67, // analyticDE_offset_1 (named)
  ABX_COUNT = 68
};
static_assert(ABX_COUNT <= MBR_SLOT_X, "Abox mod 11 block exceeds the slot's parameter block");

// aboxMod11's parameter curve (fractal_abox_mod11.cpp:96-156): the value
// added to the minimum radius^2 of the spherical fold at iteration i, in
// double precision as the reference computes it (it depends on i only)
inline MBR_HD double abox_mod11_para(const double *x, int i) {
  double para = 0.0, paraAddP0 = 0.0;
  if (x[ABX_PARA] != 0.0) {
    if (x[ABX_CP_LINEAR] != 0.0) {
      const int iterA = int(x[ABX_CP_ITERA]), iterB = int(x[ABX_CP_ITERB]), iterC = int(x[ABX_CP_ITERC]);
      para = x[ABX_CP_PARA00];
      const double temp0 = para, tempA = x[ABX_CP_PARAA], tempB = x[ABX_CP_PARAB], tempC = x[ABX_CP_PARAC];
      const double lengthAB = double(iterB - iterA);
      const double lengthBC = double(iterC - iterB);
      const double grade1 = (tempA - temp0) / double(iterA);
      const double grade2 = (tempB - tempA) / lengthAB;
      const double grade3 = (tempC - tempB) / lengthBC;
      if (i < iterA) para = temp0 + (double(i) * grade1);
      if (i < iterB && i >= iterA) para = tempA + double(i - iterA) * grade2;
      if (i >= iterB) para = tempB + double(i - iterB) * grade3;
      if (x[ABX_CP_CURVES] != 0.0) {
        double paraAdd = 0.0, paraIt;
        if (lengthAB > 2.0 * double(iterA)) {
          const double curve1 = (grade2 - grade1) / (4.0 * double(iterA));
          const double tempL = lengthAB - double(iterA);
          const double curve2 = (grade3 - grade2) / (4.0 * tempL);
          if (i < 2 * iterA) {
            paraIt = tempA - fabs(tempA - double(i));
            paraAdd = paraIt * paraIt * curve1;
          }
          if (i >= 2 * iterA && double(i) < double(iterB) + tempL) {
            paraIt = tempB - fabs(tempB * double(i));
            paraAdd = paraIt * paraIt * curve2;
          }
          para += paraAdd;
        }
      }
    }
    paraAddP0 = 0.0;
    if (x[ABX_CP_PARAB_ON] != 0.0)
      paraAddP0 = x[ABX_CP_OFFSET0] + (double(i) * x[ABX_CP_SLOPE]) + (double(i * i) * 0.001 * x[ABX_CP_SCALE]);
  }
  para += paraAddP0 + x[ABX_MINR2];
  return para;
}


// cFractalPseudoKleinianMod4 (formula/definition/fractal_pseudo_kleinian_mod4.cpp:29-145)
enum PseudoKleinianMod4X {
  P4X_SPH_INV = 0,       // transf_sphere_inversion_enabled_false
  P4X_START_X = 1,       // transf_start_iterations_X
  P4X_STOP_1 = 2,        // transf_stop_iterations_1
  P4X_OFFSET000 = 3,     // transf_offset_000 (3)
  P4X_SCALE_G1 = 6,      // transf_scaleG_1
  P4X_ADD_P000 = 7,      // transf_addition_constantP_000 (3)
  P4X_SCALE_A1 = 10,      // transf_scaleA_1
  P4X_START_M = 11,       // transf_start_iterations_M
  P4X_STOP_M = 12,        // transf_stop_iterations_M
  P4X_CM000 = 13,         // transf_constant_multiplier_000 (3)
  P4X_CSIZE = 16,         // transf_addition_constant_0777 (3)
  P4X_MINR05 = 19,        // transf_minimum_radius_05
  P4X_TWEAK005 = 20,      // analyticDE_tweak_005
  P4X_ADD000 = 21,        // transf_addition_constant (3)
  P4X_G_ON = 24,          // transf_function_enabledG_false
  P4X_START_G = 25,       // transf_start_iterations_G
  P4X_STOP_G = 26,        // transf_stop_iterations_G
  P4X_ADD_A000 = 27,      // transf_addition_constantA_000 (3)
  P4X_SCALE_NEG1 = 30,    // transf_scale_neg1
  P4X_F_ON = 31,          // transf_function_enabledF_false
  P4X_START_F = 32,       // transf_start_iterations_F
  P4X_STOP_F = 33,        // transf_stop_iterations_F
  P4X_OFFSET_A000 = 34,   // transf_offsetA_000 (3)
  P4X_N_ON = 37,          // transf_function_enabledN_false
  P4X_START_N = 38,       // transf_start_iterations_N
  P4X_STOP_N = 39,        // transf_stop_iterations_N
  P4X_SWAP_A = 40,        // transf_function_enabledA_false
  P4X_OFFSET0 = 41,       // transf_offset_0
  P4X_OFFSET_A0 = 42,     // transf_offsetA_0
  P4X_BX_F = 43,          // transf_function_enabledBx_false
  P4X_START_O = 44,       // transf_start_iterations_O
  P4X_STOP_O = 45,        // transf_stop_iterations_O
  P4X_BX = 46,            // transf_function_enabledBx
  P4X_START_P = 47,       // transf_start_iterations_P
  P4X_STOP_P = 48,        // transf_stop_iterations_P
  P4X_AX = 49,            // transf_function_enabledAx
  P4X_START_R = 50,       // transf_start_iterations_R
  P4X_STOP_R = 51,        // transf_stop_iterations_R
  P4X_OFFSET1 = 52,       // transf_offset_1
  P4X_AX_F = 53,          // transf_function_enabledAx_false
  P4X_START_RV = 54,      // transf_start_iterations_RV
  P4X_STOP_RV = 55,       // transf_stop_iterations_RV
  P4X_OFFSET_A1 = 56,     // transf_offsetA_1
  P4X_FLIP_X = 57,        // transf_function_enabledx_false
  P4X_FLIP_Y = 58,        // transf_function_enabledy_false
  P4X_FLIP_Z = 59,        // transf_function_enabledz_false
  P4X_DE_SCALE1 = 60,     // analyticDE_scale_1 (named)
  P4X_COUNT = 61
};

// cFractalPseudoKleinianStdDE (formula/definition/fractal_pseudo_kleinian_std_de.cpp:29-215)
enum PseudoKleinianStdDEX {
  PSX_P_ON = 0,        // transf_function_enabledP_false
  PSX_START_P = 1,     // transf_start_iterations_P
  PSX_STOP_P1 = 2,     // transf_stop_iterations_P1
  PSX_SCALE = 3,       // transf_scale
  PSX_CM000 = 4,       // transf_constant_multiplier_000 (3)
  PSX_R_ON = 7,        // transf_function_enabledR_false
  PSX_START_R = 8,     // transf_start_iterations_R
  PSX_STOP_R = 9,      // transf_stop_iterations_R
  PSX_ROT = 10,         // transf_rotation (10)
  PSX_T1_ON = 20,       // transf_benesi_T1_enabled_false
  PSX_START = 21,       // transf_start_iterations
  PSX_STOP_T1 = 22,     // transf_stop_iterationsT_1
  PSX_S222 = 23,        // transf_scale3D_222 (3)
  PSX_OFF200 = 26,      // transf_offset_200 (3)
  PSX_TM_ON = 29,       // transf_function_enabledx_false
  PSX_START_D = 30,     // transf_start_iterations_D
  PSX_STOP_TM1 = 31,    // transf_stop_iterationsTM_1
  PSX_S333 = 32,        // transf_scale3D_333 (3)
  PSX_ADD111 = 35,      // transf_addition_constant_111 (3)
  PSX_F_ON = 38,        // transf_function_enabledF_false
  PSX_START_F = 39,     // transf_start_iterations_F
  PSX_STOP_F = 40,      // transf_stop_iterations_F
  PSX_F_AX = 41,        // transf_function_enabledAx
  PSX_F_X = 42,         // transf_function_enabledx
  PSX_F_AY = 43,        // transf_function_enabledAy
  PSX_F_Y = 44,         // transf_function_enabledy
  PSX_F_AZ = 45,        // transf_function_enabledAz
  PSX_F_Z = 46,         // transf_function_enabledz
  PSX_OFFF000 = 47,     // transf_offsetF_000 (3)
  PSX_OFF000 = 50,      // transf_offset_000 (3)
  PSX_S111 = 53,        // transf_scale3D_111 (3)
  PSX_M_ON = 56,        // transf_function_enabled
  PSX_START_M = 57,     // transf_start_iterations_M
  PSX_STOP_M = 58,      // transf_stop_iterations_M
  PSX_CMA111 = 59,      // transf_constant_multiplierA_111 (3)
  PSX_SCALE_A1 = 62,    // transf_scaleA_1
  PSX_ADD_A000 = 63,    // transf_addition_constantA_000 (3)
  PSX_FLIP_Z = 66,      // transf_function_enabledN_false
  PSX_AW = 67,          // transf_function_enabledAw
  PSX_START_C = 68,     // transf_start_iterations_C
  PSX_STOP_C = 69,      // transf_stop_iterations_C
  PSX_CSIZE = 70,       // transf_addition_constant_0777 (3)
  PSX_SCALE_B1 = 73,    // transf_scaleB_1
  PSX_MINR05 = 74,      // transf_minimum_radius_05
  PSX_TWEAK005 = 75,    // analyticDE_tweak_005
  PSX_AYF = 76,         // transf_function_enabledAy_false
  PSX_START_B = 77,     // transf_start_iterations_B
  PSX_STOP_B = 78,      // transf_stop_iterations_B
  PSX_ADD000 = 79,      // transf_addition_constant (3)
  PSX_SCALE3 = 82,      // transf_scale_3 (named)
  PSX_COUNT = 83
};
static_assert(PSX_COUNT <= MBR_SLOT_X, "pseudo-Kleinian std DE block exceeds the slot's parameter block");

// cFractalGeneralizedFoldBox (formula/definition/fractal_generalized_fold_box.cpp:31-245):
// the keyed block, then the main rotation and the fold planes of the chosen
// polyhedron, derived on the host as sFractal's constructor and
// RecalculateFractalParams derive them (fractal.cpp:663, 713-818)
enum GeneralizedFoldBoxX {
  GFX_TYPE = 0,       // mandelbox_generalized_fold_type
  GFX_SOLID = 1,      // mandelbox_solid
  GFX_MELT = 2,       // mandelbox_melt
  GFX_MB_SCALE = 3,   // mandelbox_scale (named)
  GFX_MB_MINR = 4,    // mandelbox_folding_min_radius (named)
  GFX_MB_FIXEDR = 5,  // mandelbox_folding_fixed_radius (named)
  GFX_MB_OFFSET = 6,  // mandelbox_offset (named, 3)
  GFX_KEYED_END = 9,
  GFX_MAIN_ON = 9,    // mandelbox_main_rotation_enabled
  GFX_MAIN_ROT = 10,  // SetRotation2 of mandelbox_rotation_main (10)
  GFX_SIDES = 20,     // planes of the polyhedron
  GFX_NV = 21,        // their unit normals (up to 20 x 3)
  GFX_COUNT = 81
};
static_assert(GFX_COUNT <= MBR_SLOT_X, "generalized fold box block exceeds the slot's parameter block");

// cFractalMandelbulbPupuku (formula/definition/fractal_mandelbulb_pupuku.cpp:29-144)
enum MandelbulbPupukuX {
  PPX_P_ON = 0,        // transf_function_enabledP_false
  PPX_START_P = 1,     // transf_start_iterations_P
  PPX_STOP_P = 2,      // transf_stop_iterations_P
  PPX_CX = 3,          // transf_function_enabledCx_false
  PPX_CY = 4,          // transf_function_enabledCy_false
  PPX_CZ = 5,          // transf_function_enabledCz_false
  PPX_OFFSET_A000 = 6, // transf_offsetA_000 (3)
  PPX_T_ON = 9,        // transf_function_enabledT_false
  PPX_SW = 10,          // transf_function_enabledSw_false
  PPX_SCALE_A1 = 11,    // transf_scaleA_1
  PPX_SCALE_B1 = 12,    // transf_scaleB_1
  PPX_OFFSET1 = 13,     // transf_offset_1
  PPX_X_ON = 14,        // transf_function_enabledX_false
  PPX_START_X = 15,     // transf_start_iterations_X
  PPX_STOP_X = 16,      // transf_stop_iterations_X
  PPX_D_ON = 17,        // transf_function_enabledD_false
  PPX_B_ON = 18,        // transf_function_enabledB_false
  PPX_START_B = 19,     // transf_start_iterations_B
  PPX_STOP_B = 20,      // transf_stop_iterations_B
  PPX_SCALE_B0 = 21,    // transf_scaleB_0
  PPX_A_ON = 22,        // transf_function_enabledA_false
  PPX_START_A = 23,     // transf_start_iterations_A
  PPX_STOP_A = 24,      // transf_stop_iterations_A
  PPX_SCALE_A0 = 25,    // transf_scaleA_0
  PPX_BZ = 26,          // transf_function_enabledBz_false
  PPX_OFFSET0 = 27,     // transf_offset_0
  PPX_OFFSET000 = 28,   // transf_offset_000 (3)
  PPX_START_S = 31,     // transf_start_iterations_S
  PPX_STOP_S = 32,      // transf_stop_iterations_S
  PPX_SCALE_C1 = 33,    // transf_scaleC_1
  PPX_ADE_ON = 34,      // analyticDE_enabled_false
  PPX_ADE_OFFSET0 = 35, // analyticDE_offset_0
  PPX_C_ON = 36,        // transf_function_enabledC_false
  PPX_E_ON = 37,        // transf_function_enabledE_false
  PPX_START_E = 38,     // transf_start_iterations_E
  PPX_STOP_E = 39,      // transf_stop_iterations_E
  PPX_POWER = 40,       // power (named)
  PPX_ALPHA = 41,       // alpha_angle_offset (named)
  PPX_BETA = 42,        // beta_angle_offset (named)
  PPX_ADE_SCALE1 = 43,  // analyticDE_scale_1 (named)
  PPX_ADE_OFFSET1 = 44, // analyticDE_offset_1 (named)
  PPX_COUNT = 45
};

// cFractalDIFSHextgrid2 (formula/definition/fractal_difs_hextgrid2.cpp:30-138)
enum DIFSHextgrid2X {
  HGX_SPH_INV = 0,     // transf_sphere_inversion_enabled_false
  HGX_START_X = 1,     // transf_start_iterations_X
  HGX_STOP_1 = 2,      // transf_stop_iterations_1
  HGX_OFFSET000 = 3,   // transf_offset_000 (3)
  HGX_SCALE_G1 = 6,    // transf_scaleG_1
  HGX_ADD000 = 7,      // transf_addition_constant (3)
  HGX_SCALE_A1 = 10,    // transf_scaleA_1
  HGX_C_ON = 11,        // transf_function_enabledC_false
  HGX_START_C = 12,     // transf_start_iterations_C
  HGX_STOP_C1 = 13,     // transf_stop_iterations_C1
  HGX_OFFSET2 = 14,     // transf_offset_2
  HGX_OFFSETA2 = 15,    // transf_offsetA_2
  HGX_START_S = 16,     // transf_start_iterations_S
  HGX_STOP_S = 17,      // transf_stop_iterations_S
  HGX_SCALE2 = 18,      // transf_scale_2
  HGX_K_ON = 19,        // transf_function_enabledK_false
  HGX_START_K = 20,     // transf_start_iterations_K
  HGX_STOP_K = 21,      // transf_stop_iterations_K
  HGX_SCALE_VARY = 22,  // transf_scale_vary_0
  HGX_SCALE_C1 = 23,    // transf_scaleC_1
  HGX_OFFSET001 = 24,   // transf_offset_001 (3)
  HGX_R_ON = 27,        // transf_function_enabledR_false
  HGX_START_R = 28,     // transf_start_iterations_R
  HGX_STOP_R = 29,      // transf_stop_iterations_R
  HGX_ROT = 30,         // transf_rotation (10)
  HGX_START = 40,       // transf_start_iterations
  HGX_STOP = 41,        // transf_stop_iterations
  HGX_SCALE1 = 42,      // transf_scale_1
  HGX_SCALE_F1 = 43,    // transf_scaleF_1
  HGX_J_ON = 44,        // transf_function_enabledJ_false
  HGX_OFFSET0005 = 45,  // transf_offset_0005
  HGX_KEYED_END = 46,
  HGX_COS6 = 46,          // cos(pi / 6), host libm
  HGX_SIN6 = 47,          // sin(pi / 6), host libm
  HGX_COUNT = 48
};

#ifndef __CUDA_ARCH__
struct FormulaKey {
  const char *key;
  int kind;
  double def[3];
  int x;  // first x[] entry
};

constexpr int param_kind_size(int kind) {
  return (kind == PK_VEC3 || kind == PK_NAMED3) ? 3 : (kind == PK_ROT ? 10 : 1);
}

// true when the table's entries follow one another in x[] from 0 to end
template <int N>
constexpr bool keys_contiguous(const FormulaKey (&t)[N], int end) {
  int o = 0;
  for (int i = 0; i < N; i++) {
    if (t[i].x != o) return false;
    o += param_kind_size(t[i].kind);
  }
  return o == end;
}

constexpr FormulaKey kPseudoKleinianKeys[] = {
    {"transf_sphere_inversion_enabled_false", PK_BOOL, {0, 0, 0}, PKX_SPH_INV},
    {"transf_start_iterations_X", PK_INT, {0, 0, 0}, PKX_START_X},
    {"transf_stop_iterations_1", PK_INT, {1, 0, 0}, PKX_STOP_1},
    {"transf_offset_000", PK_VEC3, {0, 0, 0}, PKX_OFFSET000},
    {"transf_maxR2_1", PK_DOUBLE, {1, 0, 0}, PKX_MAXR2},
    {"transf_addition_constantA_000", PK_VEC3, {0, 0, 0}, PKX_ADD_A000},
    {"analyticDE_offset_0", PK_DOUBLE, {0, 0, 0}, PKX_DE_OFFSET0},
    {"transf_function_enabledP_false", PK_BOOL, {0, 0, 0}, PKX_PRISM},
    {"transf_start_iterations_P", PK_INT, {0, 0, 0}, PKX_START_P},
    {"transf_stop_iterations_P1", PK_INT, {1, 0, 0}, PKX_STOP_P1},
    {"transf_scale", PK_DOUBLE, {1, 0, 0}, PKX_SCALE},
    {"transf_constant_multiplier_000", PK_VEC3, {0, 0, 0}, PKX_CMUL000},
    {"transf_function_enabledBy_false", PK_BOOL, {0, 0, 0}, PKX_ABS_BOX},
    {"transf_start_iterations_E", PK_INT, {0, 0, 0}, PKX_START_E},
    {"transf_stop_iterations_E", PK_INT, {250, 0, 0}, PKX_STOP_E},
    {"transf_addition_constant_111", PK_VEC3, {1, 1, 1}, PKX_ADD111},
    {"transf_function_enabledBy", PK_BOOL, {1, 0, 0}, PKX_ABS_BOX_Z},
    {"transf_function_enabledBx_false", PK_BOOL, {0, 0, 0}, PKX_BOX},
    {"transf_start_iterations_A", PK_INT, {0, 0, 0}, PKX_START_A},
    {"transf_stop_iterations_A", PK_INT, {250, 0, 0}, PKX_STOP_A},
    {"transf_scale_1", PK_DOUBLE, {1, 0, 0}, PKX_SCALE1},
    {"transf_addition_constant_0777", PK_VEC3, {0.7, 0.7, 0.7}, PKX_CSIZE},
    {"transf_start_iterations_C", PK_INT, {0, 0, 0}, PKX_START_C},
    {"transf_stop_iterations_C", PK_INT, {250, 0, 0}, PKX_STOP_C},
    {"transf_minimum_radius_05", PK_DOUBLE, {0.5, 0, 0}, PKX_MINR05},
    {"transf_function_enabledN_false", PK_BOOL, {0, 0, 0}, PKX_FLIP_Z},
    {"transf_function_enabledw_false", PK_BOOL, {0, 0, 0}, PKX_FLIP_W},
    {"analyticDE_tweak_005", PK_DOUBLE, {0.05, 0, 0}, PKX_TWEAK005},
    {"transf_function_enabledR_false", PK_BOOL, {0, 0, 0}, PKX_ROT_ON},
    {"transf_start_iterations_R", PK_INT, {0, 0, 0}, PKX_START_R},
    {"transf_stop_iterations_R", PK_INT, {250, 0, 0}, PKX_STOP_R},
    {"transf_rotation", PK_ROT, {0, 0, 0}, PKX_ROT},
    {"transf_addition_constant", PK_VEC3, {0, 0, 0}, PKX_ADD000},
    {"mandelbox_folding_limit", PK_NAMED, {NF_MB_LIMIT, 0, 0}, PKX_MB_LIMIT},
    {"mandelbox_folding_value", PK_NAMED, {NF_MB_VALUE, 0, 0}, PKX_MB_VALUE},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1, 0, 0}, PKX_DE_SCALE1},
};
static_assert(keys_contiguous(kPseudoKleinianKeys, PKX_COUNT), "pseudo-Kleinian keys and x[] layout disagree");

constexpr FormulaKey kBoxFoldBulbPow2Keys[] = {
    {"boxfold_bulbpow2_folding_factor", PK_DOUBLE, {2, 0, 0}, BFX_FOLD},
    {"boxfold_bulbpow2_z_factor", PK_DOUBLE, {5, 0, 0}, BFX_ZFACTOR},
    {"analyticDE_enabled_false", PK_BOOL, {0, 0, 0}, BFX_ADE_ON},
    {"analyticDE_offset_2", PK_DOUBLE, {1, 0, 0}, BFX_ADE_OFFSET2},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1, 0, 0}, BFX_ADE_SCALE1},
    {"analyticDE_offset_1", PK_NAMED, {NF_ADE_OFFSET1, 0, 0}, BFX_ADE_OFFSET1},
};
static_assert(keys_contiguous(kBoxFoldBulbPow2Keys, BFX_COUNT), "box fold bulb pow 2 keys and layout disagree");

constexpr FormulaKey kMengerMod1Keys[] = {
    {"transf_constant_multiplier_111", PK_VEC3, {1, 1, 1}, MMX_CM111},
    {"transf_rotation_enabled", PK_BOOL, {0, 0, 0}, MMX_ROT_ON},
    {"transf_start_iterations", PK_INT, {0, 0, 0}, MMX_START},
    {"transf_stop_iterations", PK_INT, {250, 0, 0}, MMX_STOP},
    {"transf_rotation", PK_ROT, {0, 0, 0}, MMX_ROT},
    {"transf_scaleD_1", PK_DOUBLE, {1, 0, 0}, MMX_SCALED1},
    {"transf_offset_1", PK_DOUBLE, {1, 0, 0}, MMX_OFFSET1},
    {"transf_addition_constant", PK_VEC3, {0, 0, 0}, MMX_ADD000},
    {"transf_function_enabledx_false", PK_BOOL, {0, 0, 0}, MMX_BOX_OFF},
    {"transf_start_iterations_A", PK_INT, {0, 0, 0}, MMX_START_A},
    {"transf_stop_iterations_A", PK_INT, {250, 0, 0}, MMX_STOP_A},
    {"transf_addition_constantA_000", PK_VEC3, {0, 0, 0}, MMX_ADD_A000},
    {"transf_function_enabledA_false", PK_BOOL, {0, 0, 0}, MMX_AVG_SCALE},
    {"transf_function_enabled_false", PK_BOOL, {0, 0, 0}, MMX_BLEND},
    {"transf_int_A", PK_INT, {0, 0, 0}, MMX_INT_A},
    {"transf_int_B", PK_INT, {0, 0, 0}, MMX_INT_B},
    {"transf_scale_1", PK_DOUBLE, {1, 0, 0}, MMX_SCALE1},
    {"transf_offset", PK_DOUBLE, {0, 0, 0}, MMX_OFFSET},
    {"transf_offset_0", PK_DOUBLE, {0, 0, 0}, MMX_OFFSET0},
    {"transf_scale_3", PK_NAMED, {NF_SCALE3, 0, 0}, MMX_SCALE3},
};
static_assert(keys_contiguous(kMengerMod1Keys, MMX_COUNT), "Menger mod 1 keys and layout disagree");

constexpr FormulaKey kBoxFoldBulbPow2V2Keys[] = {
    {"transf_addition_constant_111", PK_VEC3, {1, 1, 1}, B2X_ADD111},
    {"transf_start_iterations_B", PK_INT, {0, 0, 0}, B2X_START_B},
    {"transf_stop_iterations_B", PK_INT, {250, 0, 0}, B2X_STOP_B},
    {"transf_start_iterations_S", PK_INT, {0, 0, 0}, B2X_START_S},
    {"transf_stop_iterations_S", PK_INT, {250, 0, 0}, B2X_STOP_S},
    {"transf_minR2_p25", PK_DOUBLE, {0.25, 0, 0}, B2X_MINR2},
    {"transf_maxR2_1", PK_DOUBLE, {1, 0, 0}, B2X_MAXR2},
    {"transf_start_iterations_C", PK_INT, {0, 0, 0}, B2X_START_C},
    {"transf_stop_iterations_C", PK_INT, {250, 0, 0}, B2X_STOP_C},
    {"transf_scale", PK_DOUBLE, {1, 0, 0}, B2X_SCALE},
    {"transf_start_iterations_X", PK_INT, {0, 0, 0}, B2X_START_X},
    {"transf_stop_iterations_X", PK_INT, {250, 0, 0}, B2X_STOP_X},
    {"transf_scale_vary_0", PK_DOUBLE, {0, 0, 0}, B2X_SCALE_VARY},
    {"transf_scaleB_1", PK_DOUBLE, {1, 0, 0}, B2X_SCALE_B1},
    {"transf_function_enabledM_false", PK_BOOL, {0, 0, 0}, B2X_VARY_M},
    {"transf_start_iterations_A", PK_INT, {0, 0, 0}, B2X_START_A},
    {"transf_stop_iterations_A", PK_INT, {250, 0, 0}, B2X_STOP_A},
    {"boxfold_bulbpow2_z_factor", PK_DOUBLE, {5, 0, 0}, B2X_ZFACTOR},
    {"analyticDE_offset_2", PK_DOUBLE, {1, 0, 0}, B2X_ADE_OFFSET2},
    {"mandelbox_offset", PK_NAMED3, {NF_MB_OFFSET, 0, 0}, B2X_MB_OFFSET},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1, 0, 0}, B2X_ADE_SCALE1},
    {"analyticDE_offset_1", PK_NAMED, {NF_ADE_OFFSET1, 0, 0}, B2X_ADE_OFFSET1},
};
static_assert(keys_contiguous(kBoxFoldBulbPow2V2Keys, B2X_COUNT), "box fold bulb pow 2 V2 keys and layout disagree");

constexpr FormulaKey kAboxMod11Keys[] = {
    {"mandelbox_vary_scale_vary", PK_DOUBLE, {0, 0, 0}, ABX_SCALE_VARY},
    {"transf_addition_constant_111", PK_VEC3, {1, 1, 1}, ABX_ADD111},
    {"transf_start_iterations_B", PK_INT, {0, 0, 0}, ABX_START_B},
    {"transf_stop_iterations_B", PK_INT, {250, 0, 0}, ABX_STOP_B},
    {"transf_function_enabled", PK_BOOL, {1, 0, 0}, ABX_FOLD_Z},
    {"transf_function_enabled_false", PK_BOOL, {0, 0, 0}, ABX_FOLD_D},
    {"transf_start_iterations_D", PK_INT, {0, 0, 0}, ABX_START_D},
    {"transf_stop_iterations_D1", PK_INT, {1, 0, 0}, ABX_STOP_D1},
    {"transf_scale3D_000", PK_VEC3, {0, 0, 0}, ABX_SCALE3D},
    {"transf_function_enabledSw_false", PK_BOOL, {0, 0, 0}, ABX_SWAP},
    {"transf_start_iterations_S", PK_INT, {0, 0, 0}, ABX_START_S},
    {"transf_stop_iterations_S", PK_INT, {250, 0, 0}, ABX_STOP_S},
    {"transf_function_enabledy_false", PK_BOOL, {0, 0, 0}, ABX_PARA},
    {"Cpara_enabledLinear", PK_BOOL, {1, 0, 0}, ABX_CP_LINEAR},
    {"Cpara_para00", PK_DOUBLE, {0, 0, 0}, ABX_CP_PARA00},
    {"Cpara_paraA", PK_DOUBLE, {1, 0, 0}, ABX_CP_PARAA},
    {"Cpara_paraB", PK_DOUBLE, {1, 0, 0}, ABX_CP_PARAB},
    {"Cpara_paraC", PK_DOUBLE, {1, 0, 0}, ABX_CP_PARAC},
    {"Cpara_iterA", PK_INT, {250, 0, 0}, ABX_CP_ITERA},
    {"Cpara_iterB", PK_INT, {250, 0, 0}, ABX_CP_ITERB},
    {"Cpara_iterC", PK_INT, {250, 0, 0}, ABX_CP_ITERC},
    {"Cpara_enabledCurves", PK_BOOL, {1, 0, 0}, ABX_CP_CURVES},
    {"Cpara_enabledParab_false", PK_BOOL, {0, 0, 0}, ABX_CP_PARAB_ON},
    {"Cpara_parab_offset0", PK_DOUBLE, {0, 0, 0}, ABX_CP_OFFSET0},
    {"Cpara_parab_slope", PK_DOUBLE, {0, 0, 0}, ABX_CP_SLOPE},
    {"Cpara_parab_scale", PK_DOUBLE, {0, 0, 0}, ABX_CP_SCALE},
    {"transf_minR2_p25", PK_DOUBLE, {0.25, 0, 0}, ABX_MINR2},
    {"transf_maxR2_1", PK_DOUBLE, {1, 0, 0}, ABX_MAXR2},
    {"transf_start_iterations_A", PK_INT, {0, 0, 0}, ABX_START_A},
    {"transf_stop_iterations_A", PK_INT, {250, 0, 0}, ABX_STOP_A},
    {"analyticDE_enabled_false", PK_BOOL, {0, 0, 0}, ABX_ADE_ON},
    {"transf_addition_constant", PK_VEC3, {0, 0, 0}, ABX_ADD000},
    {"transf_addCpixel_enabled_false", PK_BOOL, {0, 0, 0}, ABX_ADDC},
    {"transf_start_iterations_E", PK_INT, {0, 0, 0}, ABX_START_E},
    {"transf_stop_iterations_E", PK_INT, {250, 0, 0}, ABX_STOP_E},
    {"transf_alternate_enabled_false", PK_BOOL, {0, 0, 0}, ABX_ALTERNATE},
    {"mandelbulbMulti_order_of_xyz", PK_INT, {0, 0, 0}, ABX_ORDER},
    {"transf_constant_multiplier_111", PK_VEC3, {1, 1, 1}, ABX_CM111},
    {"transf_rotation_enabled", PK_BOOL, {0, 0, 0}, ABX_ROT_ON},
    {"transf_start_iterations_R", PK_INT, {0, 0, 0}, ABX_START_R},
    {"transf_stop_iterations_R", PK_INT, {250, 0, 0}, ABX_STOP_R},
    {"transf_rotation", PK_ROT, {0, 0, 0}, ABX_ROT},
    {"transf_start_iterations_C", PK_INT, {0, 0, 0}, ABX_START_C},
    {"transf_stop_iterations_C1", PK_INT, {1, 0, 0}, ABX_STOP_C1},
    {"transf_scaleG_1", PK_DOUBLE, {1, 0, 0}, ABX_SCALE_G1},
    {"mandelbox_offset", PK_NAMED3, {NF_MB_OFFSET, 0, 0}, ABX_MB_OFFSET},
    {"mandelbox_scale", PK_NAMED, {NF_MB_SCALE, 0, 0}, ABX_MB_SCALE},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1, 0, 0}, ABX_ADE_SCALE1},
    {"analyticDE_offset_1", PK_NAMED, {NF_ADE_OFFSET1, 0, 0}, ABX_ADE_OFFSET1},
};
static_assert(keys_contiguous(kAboxMod11Keys, ABX_COUNT), "Abox mod 11 keys and layout disagree");

constexpr FormulaKey kPseudoKleinianMod4Keys[] = {
    {"transf_sphere_inversion_enabled_false", PK_BOOL, {0,0,0}, P4X_SPH_INV},
    {"transf_start_iterations_X", PK_INT, {0,0,0}, P4X_START_X},
    {"transf_stop_iterations_1", PK_INT, {1,0,0}, P4X_STOP_1},
    {"transf_offset_000", PK_VEC3, {0,0,0}, P4X_OFFSET000},
    {"transf_scaleG_1", PK_DOUBLE, {1,0,0}, P4X_SCALE_G1},
    {"transf_addition_constantP_000", PK_VEC3, {0,0,0}, P4X_ADD_P000},
    {"transf_scaleA_1", PK_DOUBLE, {1,0,0}, P4X_SCALE_A1},
    {"transf_start_iterations_M", PK_INT, {0,0,0}, P4X_START_M},
    {"transf_stop_iterations_M", PK_INT, {250,0,0}, P4X_STOP_M},
    {"transf_constant_multiplier_000", PK_VEC3, {0,0,0}, P4X_CM000},
    {"transf_addition_constant_0777", PK_VEC3, {0.7,0.7,0.7}, P4X_CSIZE},
    {"transf_minimum_radius_05", PK_DOUBLE, {0.5,0,0}, P4X_MINR05},
    {"analyticDE_tweak_005", PK_DOUBLE, {0.05,0,0}, P4X_TWEAK005},
    {"transf_addition_constant", PK_VEC3, {0,0,0}, P4X_ADD000},
    {"transf_function_enabledG_false", PK_BOOL, {0,0,0}, P4X_G_ON},
    {"transf_start_iterations_G", PK_INT, {0,0,0}, P4X_START_G},
    {"transf_stop_iterations_G", PK_INT, {250,0,0}, P4X_STOP_G},
    {"transf_addition_constantA_000", PK_VEC3, {0,0,0}, P4X_ADD_A000},
    {"transf_scale_neg1", PK_DOUBLE, {-1,0,0}, P4X_SCALE_NEG1},
    {"transf_function_enabledF_false", PK_BOOL, {0,0,0}, P4X_F_ON},
    {"transf_start_iterations_F", PK_INT, {0,0,0}, P4X_START_F},
    {"transf_stop_iterations_F", PK_INT, {250,0,0}, P4X_STOP_F},
    {"transf_offsetA_000", PK_VEC3, {0,0,0}, P4X_OFFSET_A000},
    {"transf_function_enabledN_false", PK_BOOL, {0,0,0}, P4X_N_ON},
    {"transf_start_iterations_N", PK_INT, {0,0,0}, P4X_START_N},
    {"transf_stop_iterations_N", PK_INT, {250,0,0}, P4X_STOP_N},
    {"transf_function_enabledA_false", PK_BOOL, {0,0,0}, P4X_SWAP_A},
    {"transf_offset_0", PK_DOUBLE, {0,0,0}, P4X_OFFSET0},
    {"transf_offsetA_0", PK_DOUBLE, {0,0,0}, P4X_OFFSET_A0},
    {"transf_function_enabledBx_false", PK_BOOL, {0,0,0}, P4X_BX_F},
    {"transf_start_iterations_O", PK_INT, {0,0,0}, P4X_START_O},
    {"transf_stop_iterations_O", PK_INT, {250,0,0}, P4X_STOP_O},
    {"transf_function_enabledBx", PK_BOOL, {1,0,0}, P4X_BX},
    {"transf_start_iterations_P", PK_INT, {0,0,0}, P4X_START_P},
    {"transf_stop_iterations_P", PK_INT, {250,0,0}, P4X_STOP_P},
    {"transf_function_enabledAx", PK_BOOL, {1,0,0}, P4X_AX},
    {"transf_start_iterations_R", PK_INT, {0,0,0}, P4X_START_R},
    {"transf_stop_iterations_R", PK_INT, {250,0,0}, P4X_STOP_R},
    {"transf_offset_1", PK_DOUBLE, {1,0,0}, P4X_OFFSET1},
    {"transf_function_enabledAx_false", PK_BOOL, {0,0,0}, P4X_AX_F},
    {"transf_start_iterations_RV", PK_INT, {0,0,0}, P4X_START_RV},
    {"transf_stop_iterations_RV", PK_INT, {250,0,0}, P4X_STOP_RV},
    {"transf_offsetA_1", PK_DOUBLE, {1,0,0}, P4X_OFFSET_A1},
    {"transf_function_enabledx_false", PK_BOOL, {0,0,0}, P4X_FLIP_X},
    {"transf_function_enabledy_false", PK_BOOL, {0,0,0}, P4X_FLIP_Y},
    {"transf_function_enabledz_false", PK_BOOL, {0,0,0}, P4X_FLIP_Z},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1,0,0}, P4X_DE_SCALE1},
};
static_assert(keys_contiguous(kPseudoKleinianMod4Keys, P4X_COUNT), "pseudo-Kleinian mod 4 keys and layout disagree");

constexpr FormulaKey kPseudoKleinianStdDEKeys[] = {
    {"transf_function_enabledP_false", PK_BOOL, {0,0,0}, PSX_P_ON},
    {"transf_start_iterations_P", PK_INT, {0,0,0}, PSX_START_P},
    {"transf_stop_iterations_P1", PK_INT, {1,0,0}, PSX_STOP_P1},
    {"transf_scale", PK_DOUBLE, {1,0,0}, PSX_SCALE},
    {"transf_constant_multiplier_000", PK_VEC3, {0,0,0}, PSX_CM000},
    {"transf_function_enabledR_false", PK_BOOL, {0,0,0}, PSX_R_ON},
    {"transf_start_iterations_R", PK_INT, {0,0,0}, PSX_START_R},
    {"transf_stop_iterations_R", PK_INT, {250,0,0}, PSX_STOP_R},
    {"transf_rotation", PK_ROT, {0,0,0}, PSX_ROT},
    {"transf_benesi_T1_enabled_false", PK_BOOL, {0,0,0}, PSX_T1_ON},
    {"transf_start_iterations", PK_INT, {0,0,0}, PSX_START},
    {"transf_stop_iterationsT_1", PK_INT, {1,0,0}, PSX_STOP_T1},
    {"transf_scale3D_222", PK_VEC3, {2,2,2}, PSX_S222},
    {"transf_offset_200", PK_VEC3, {2,0,0}, PSX_OFF200},
    {"transf_function_enabledx_false", PK_BOOL, {0,0,0}, PSX_TM_ON},
    {"transf_start_iterations_D", PK_INT, {0,0,0}, PSX_START_D},
    {"transf_stop_iterationsTM_1", PK_INT, {1,0,0}, PSX_STOP_TM1},
    {"transf_scale3D_333", PK_VEC3, {3,3,3}, PSX_S333},
    {"transf_addition_constant_111", PK_VEC3, {1,1,1}, PSX_ADD111},
    {"transf_function_enabledF_false", PK_BOOL, {0,0,0}, PSX_F_ON},
    {"transf_start_iterations_F", PK_INT, {0,0,0}, PSX_START_F},
    {"transf_stop_iterations_F", PK_INT, {250,0,0}, PSX_STOP_F},
    {"transf_function_enabledAx", PK_BOOL, {1,0,0}, PSX_F_AX},
    {"transf_function_enabledx", PK_BOOL, {1,0,0}, PSX_F_X},
    {"transf_function_enabledAy", PK_BOOL, {1,0,0}, PSX_F_AY},
    {"transf_function_enabledy", PK_BOOL, {1,0,0}, PSX_F_Y},
    {"transf_function_enabledAz", PK_BOOL, {1,0,0}, PSX_F_AZ},
    {"transf_function_enabledz", PK_BOOL, {1,0,0}, PSX_F_Z},
    {"transf_offsetF_000", PK_VEC3, {0,0,0}, PSX_OFFF000},
    {"transf_offset_000", PK_VEC3, {0,0,0}, PSX_OFF000},
    {"transf_scale3D_111", PK_VEC3, {1,1,1}, PSX_S111},
    {"transf_function_enabled", PK_BOOL, {1,0,0}, PSX_M_ON},
    {"transf_start_iterations_M", PK_INT, {0,0,0}, PSX_START_M},
    {"transf_stop_iterations_M", PK_INT, {250,0,0}, PSX_STOP_M},
    {"transf_constant_multiplierA_111", PK_VEC3, {1,1,1}, PSX_CMA111},
    {"transf_scaleA_1", PK_DOUBLE, {1,0,0}, PSX_SCALE_A1},
    {"transf_addition_constantA_000", PK_VEC3, {0,0,0}, PSX_ADD_A000},
    {"transf_function_enabledN_false", PK_BOOL, {0,0,0}, PSX_FLIP_Z},
    {"transf_function_enabledAw", PK_BOOL, {1,0,0}, PSX_AW},
    {"transf_start_iterations_C", PK_INT, {0,0,0}, PSX_START_C},
    {"transf_stop_iterations_C", PK_INT, {250,0,0}, PSX_STOP_C},
    {"transf_addition_constant_0777", PK_VEC3, {0.7,0.7,0.7}, PSX_CSIZE},
    {"transf_scaleB_1", PK_DOUBLE, {1,0,0}, PSX_SCALE_B1},
    {"transf_minimum_radius_05", PK_DOUBLE, {0.5,0,0}, PSX_MINR05},
    {"analyticDE_tweak_005", PK_DOUBLE, {0.05,0,0}, PSX_TWEAK005},
    {"transf_function_enabledAy_false", PK_BOOL, {0,0,0}, PSX_AYF},
    {"transf_start_iterations_B", PK_INT, {0,0,0}, PSX_START_B},
    {"transf_stop_iterations_B", PK_INT, {250,0,0}, PSX_STOP_B},
    {"transf_addition_constant", PK_VEC3, {0,0,0}, PSX_ADD000},
    {"transf_scale_3", PK_NAMED, {NF_SCALE3,0,0}, PSX_SCALE3},
};
static_assert(keys_contiguous(kPseudoKleinianStdDEKeys, PSX_COUNT), "pseudo-Kleinian std DE keys and layout disagree");

constexpr FormulaKey kGeneralizedFoldBoxKeys[] = {
    {"mandelbox_generalized_fold_type", PK_INT, {0, 0, 0}, GFX_TYPE},
    {"mandelbox_solid", PK_DOUBLE, {1, 0, 0}, GFX_SOLID},
    {"mandelbox_melt", PK_DOUBLE, {0, 0, 0}, GFX_MELT},
    {"mandelbox_scale", PK_NAMED, {NF_MB_SCALE, 0, 0}, GFX_MB_SCALE},
    {"mandelbox_folding_min_radius", PK_NAMED, {NF_MB_MIN_R, 0, 0}, GFX_MB_MINR},
    {"mandelbox_folding_fixed_radius", PK_NAMED, {NF_MB_FIXED_R, 0, 0}, GFX_MB_FIXEDR},
    {"mandelbox_offset", PK_NAMED3, {NF_MB_OFFSET, 0, 0}, GFX_MB_OFFSET},
};
static_assert(keys_contiguous(kGeneralizedFoldBoxKeys, GFX_KEYED_END), "generalized fold box keys and layout disagree");

// The fold planes of enumGeneralizedFoldBoxType `type` (fractal.h:66-76) into
// nv (x, y, z per plane), as sFractal's constructor builds them
// (fractal.cpp:713-818); returns the number of planes.  An unknown type is
// the tetrahedron, the switch's default.
inline int generalized_fold_box_planes(int type, double *nv) {
  const double pi = 3.14159265358979323846;
  const double s = 1.0 / std::sqrt(3.0);
  const double tet[8][3] = {{s, s, -s}, {s, -s, s}, {-s, s, s}, {-s, -s, -s},
                            {s, s, s}, {-s, -s, s}, {-s, s, -s}, {s, -s, -s}};
  const double cube[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  int n = 0;
  auto put = [&](double a, double b, double c) {
    nv[3 * n] = a;
    nv[3 * n + 1] = b;
    nv[3 * n + 2] = c;
    n++;
  };
  const double aa = ((1.0 + std::sqrt(5.0)) / 2.0);
  const double bb = (1.0 / std::sqrt(aa * aa + 1.0));
  const double ff = std::sqrt(aa * aa + 1.0 / (aa * aa));
  const double cc = aa / ff;
  const double dd = 1.0 / aa / ff;
  switch (type) {
    case 1:  // cube
      for (int i = 0; i < 6; i++) put(cube[i][0], cube[i][1], cube[i][2]);
      break;
    case 2:  // octahedron
      for (int i = 0; i < 8; i++) put(tet[i][0], tet[i][1], tet[i][2]);
      break;
    case 3:  // dodecahedron
      put(0, bb, aa * bb); put(0, bb, -aa * bb); put(0, -bb, aa * bb); put(0, -bb, -aa * bb);
      put(bb, aa * bb, 0); put(bb, -aa * bb, 0); put(-bb, aa * bb, 0); put(-bb, -aa * bb, 0);
      put(aa * bb, 0, bb); put(-aa * bb, 0, bb); put(aa * bb, 0, -bb); put(-aa * bb, 0, -bb);
      break;
    case 4:  // octahedron and cube
      for (int i = 0; i < 8; i++) put(tet[i][0], tet[i][1], tet[i][2]);
      for (int i = 0; i < 6; i++) put(cube[i][0], cube[i][1], cube[i][2]);
      break;
    case 5:  // icosahedron
      for (int i = 0; i < 8; i++) put(tet[i][0], tet[i][1], tet[i][2]);
      put(0, dd, cc); put(0, dd, -cc); put(0, -dd, cc); put(0, -dd, -cc);
      put(cc, 0, dd); put(cc, 0, -dd); put(-cc, 0, dd); put(-cc, 0, -dd);
      put(dd, cc, 0); put(dd, -cc, 0); put(-dd, cc, 0); put(-dd, -cc, 0);
      break;
    case 6: {  // hexagonal prism
      const double tha = pi * 2.0 / 6.0;
      put(0, 0, 1); put(0, 0, -1);
      for (int k = 0; k < 6; k++) put(std::cos(tha * k), std::sin(tha * k), 0);
      break;
    }
    case 7: {  // pentagonal prism
      const double tha5 = pi * 2.0 / 5.0;
      put(0, 0, 1); put(0, 0, -1);
      for (int k = 0; k < 5; k++) put(std::cos(tha5 * k), std::sin(tha5 * k), 0);
      break;
    }
    default:  // tetrahedron
      for (int i = 0; i < 4; i++) put(tet[i][0], tet[i][1], tet[i][2]);
      break;
  }
  return n;
}

constexpr FormulaKey kMandelbulbPupukuKeys[] = {
    {"transf_function_enabledP_false", PK_BOOL, {0,0,0}, PPX_P_ON},
    {"transf_start_iterations_P", PK_INT, {0,0,0}, PPX_START_P},
    {"transf_stop_iterations_P", PK_INT, {250,0,0}, PPX_STOP_P},
    {"transf_function_enabledCx_false", PK_BOOL, {0,0,0}, PPX_CX},
    {"transf_function_enabledCy_false", PK_BOOL, {0,0,0}, PPX_CY},
    {"transf_function_enabledCz_false", PK_BOOL, {0,0,0}, PPX_CZ},
    {"transf_offsetA_000", PK_VEC3, {0,0,0}, PPX_OFFSET_A000},
    {"transf_function_enabledT_false", PK_BOOL, {0,0,0}, PPX_T_ON},
    {"transf_function_enabledSw_false", PK_BOOL, {0,0,0}, PPX_SW},
    {"transf_scaleA_1", PK_DOUBLE, {1,0,0}, PPX_SCALE_A1},
    {"transf_scaleB_1", PK_DOUBLE, {1,0,0}, PPX_SCALE_B1},
    {"transf_offset_1", PK_DOUBLE, {1,0,0}, PPX_OFFSET1},
    {"transf_function_enabledX_false", PK_BOOL, {0,0,0}, PPX_X_ON},
    {"transf_start_iterations_X", PK_INT, {0,0,0}, PPX_START_X},
    {"transf_stop_iterations_X", PK_INT, {250,0,0}, PPX_STOP_X},
    {"transf_function_enabledD_false", PK_BOOL, {0,0,0}, PPX_D_ON},
    {"transf_function_enabledB_false", PK_BOOL, {0,0,0}, PPX_B_ON},
    {"transf_start_iterations_B", PK_INT, {0,0,0}, PPX_START_B},
    {"transf_stop_iterations_B", PK_INT, {250,0,0}, PPX_STOP_B},
    {"transf_scaleB_0", PK_DOUBLE, {0,0,0}, PPX_SCALE_B0},
    {"transf_function_enabledA_false", PK_BOOL, {0,0,0}, PPX_A_ON},
    {"transf_start_iterations_A", PK_INT, {0,0,0}, PPX_START_A},
    {"transf_stop_iterations_A", PK_INT, {250,0,0}, PPX_STOP_A},
    {"transf_scaleA_0", PK_DOUBLE, {0,0,0}, PPX_SCALE_A0},
    {"transf_function_enabledBz_false", PK_BOOL, {0,0,0}, PPX_BZ},
    {"transf_offset_0", PK_DOUBLE, {0,0,0}, PPX_OFFSET0},
    {"transf_offset_000", PK_VEC3, {0,0,0}, PPX_OFFSET000},
    {"transf_start_iterations_S", PK_INT, {0,0,0}, PPX_START_S},
    {"transf_stop_iterations_S", PK_INT, {250,0,0}, PPX_STOP_S},
    {"transf_scaleC_1", PK_DOUBLE, {1,0,0}, PPX_SCALE_C1},
    {"analyticDE_enabled_false", PK_BOOL, {0,0,0}, PPX_ADE_ON},
    {"analyticDE_offset_0", PK_DOUBLE, {0,0,0}, PPX_ADE_OFFSET0},
    {"transf_function_enabledC_false", PK_BOOL, {0,0,0}, PPX_C_ON},
    {"transf_function_enabledE_false", PK_BOOL, {0,0,0}, PPX_E_ON},
    {"transf_start_iterations_E", PK_INT, {0,0,0}, PPX_START_E},
    {"transf_stop_iterations_E", PK_INT, {250,0,0}, PPX_STOP_E},
    {"power", PK_NAMED, {NF_POWER,0,0}, PPX_POWER},
    {"alpha_angle_offset", PK_NAMED, {NF_ALPHA,0,0}, PPX_ALPHA},
    {"beta_angle_offset", PK_NAMED, {NF_BETA,0,0}, PPX_BETA},
    {"analyticDE_scale_1", PK_NAMED, {NF_ADE_SCALE1,0,0}, PPX_ADE_SCALE1},
    {"analyticDE_offset_1", PK_NAMED, {NF_ADE_OFFSET1,0,0}, PPX_ADE_OFFSET1},
};
static_assert(keys_contiguous(kMandelbulbPupukuKeys, PPX_COUNT), "Mandelbulb Pupuku keys and layout disagree");

constexpr FormulaKey kDIFSHextgrid2Keys[] = {
    {"transf_sphere_inversion_enabled_false", PK_BOOL, {0,0,0}, HGX_SPH_INV},
    {"transf_start_iterations_X", PK_INT, {0,0,0}, HGX_START_X},
    {"transf_stop_iterations_1", PK_INT, {1,0,0}, HGX_STOP_1},
    {"transf_offset_000", PK_VEC3, {0,0,0}, HGX_OFFSET000},
    {"transf_scaleG_1", PK_DOUBLE, {1,0,0}, HGX_SCALE_G1},
    {"transf_addition_constant", PK_VEC3, {0,0,0}, HGX_ADD000},
    {"transf_scaleA_1", PK_DOUBLE, {1,0,0}, HGX_SCALE_A1},
    {"transf_function_enabledC_false", PK_BOOL, {0,0,0}, HGX_C_ON},
    {"transf_start_iterations_C", PK_INT, {0,0,0}, HGX_START_C},
    {"transf_stop_iterations_C1", PK_INT, {1,0,0}, HGX_STOP_C1},
    {"transf_offset_2", PK_DOUBLE, {2,0,0}, HGX_OFFSET2},
    {"transf_offsetA_2", PK_DOUBLE, {2,0,0}, HGX_OFFSETA2},
    {"transf_start_iterations_S", PK_INT, {0,0,0}, HGX_START_S},
    {"transf_stop_iterations_S", PK_INT, {250,0,0}, HGX_STOP_S},
    {"transf_scale_2", PK_DOUBLE, {2,0,0}, HGX_SCALE2},
    {"transf_function_enabledK_false", PK_BOOL, {0,0,0}, HGX_K_ON},
    {"transf_start_iterations_K", PK_INT, {0,0,0}, HGX_START_K},
    {"transf_stop_iterations_K", PK_INT, {250,0,0}, HGX_STOP_K},
    {"transf_scale_vary_0", PK_DOUBLE, {0,0,0}, HGX_SCALE_VARY},
    {"transf_scaleC_1", PK_DOUBLE, {1,0,0}, HGX_SCALE_C1},
    {"transf_offset_001", PK_VEC3, {0,0,1}, HGX_OFFSET001},
    {"transf_function_enabledR_false", PK_BOOL, {0,0,0}, HGX_R_ON},
    {"transf_start_iterations_R", PK_INT, {0,0,0}, HGX_START_R},
    {"transf_stop_iterations_R", PK_INT, {250,0,0}, HGX_STOP_R},
    {"transf_rotation", PK_ROT, {0,0,0}, HGX_ROT},
    {"transf_start_iterations", PK_INT, {0,0,0}, HGX_START},
    {"transf_stop_iterations", PK_INT, {250,0,0}, HGX_STOP},
    {"transf_scale_1", PK_DOUBLE, {1,0,0}, HGX_SCALE1},
    {"transf_scaleF_1", PK_DOUBLE, {1,0,0}, HGX_SCALE_F1},
    {"transf_function_enabledJ_false", PK_BOOL, {0,0,0}, HGX_J_ON},
    {"transf_offset_0005", PK_DOUBLE, {0.005,0,0}, HGX_OFFSET0005},
};
static_assert(keys_contiguous(kDIFSHextgrid2Keys, HGX_KEYED_END), "DIFS hextgrid2 keys and layout disagree");

struct KeyTable {
  const FormulaKey *keys;
  int n;
};

// the key table of a keyed formula; n = 0 for the others
inline KeyTable formula_keys(int formula) {
  switch (formula) {
    case MBR_FORMULA_PSEUDO_KLEINIAN:
      return {kPseudoKleinianKeys, int(sizeof(kPseudoKleinianKeys) / sizeof(kPseudoKleinianKeys[0]))};
    case MBR_FORMULA_BOX_FOLD_BULB_POW2:
      return {kBoxFoldBulbPow2Keys, int(sizeof(kBoxFoldBulbPow2Keys) / sizeof(kBoxFoldBulbPow2Keys[0]))};
    case MBR_FORMULA_MENGER_MOD1:
      return {kMengerMod1Keys, int(sizeof(kMengerMod1Keys) / sizeof(kMengerMod1Keys[0]))};
    case MBR_FORMULA_BOX_FOLD_BULB_POW2_V2:
      return {kBoxFoldBulbPow2V2Keys, int(sizeof(kBoxFoldBulbPow2V2Keys) / sizeof(kBoxFoldBulbPow2V2Keys[0]))};
    case MBR_FORMULA_ABOX_MOD11:
      return {kAboxMod11Keys, int(sizeof(kAboxMod11Keys) / sizeof(kAboxMod11Keys[0]))};
    case MBR_FORMULA_PSEUDO_KLEINIAN_MOD4:
      return {kPseudoKleinianMod4Keys, int(sizeof(kPseudoKleinianMod4Keys) / sizeof(kPseudoKleinianMod4Keys[0]))};
    case MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE:
      return {kPseudoKleinianStdDEKeys, int(sizeof(kPseudoKleinianStdDEKeys) / sizeof(kPseudoKleinianStdDEKeys[0]))};
    case MBR_FORMULA_GENERALIZED_FOLD_BOX:
      return {kGeneralizedFoldBoxKeys, int(sizeof(kGeneralizedFoldBoxKeys) / sizeof(kGeneralizedFoldBoxKeys[0]))};
    case MBR_FORMULA_MANDELBULB_PUPUKU:
      return {kMandelbulbPupukuKeys, int(sizeof(kMandelbulbPupukuKeys) / sizeof(kMandelbulbPupukuKeys[0]))};
    case MBR_FORMULA_DIFS_HEXTGRID2:
      return {kDIFSHextgrid2Keys, int(sizeof(kDIFSHextgrid2Keys) / sizeof(kDIFSHextgrid2Keys[0]))};
    default: return {nullptr, 0};
  }
}

// The entry of `key` in the table, or -1 (also for a NAMED entry, whose
// value comes from its mbr_fractal field).
inline int find_key(const KeyTable &t, const char *key) {
  for (int i = 0; i < t.n; i++) {
    if (t.keys[i].kind == PK_NAMED || t.keys[i].kind == PK_NAMED3) continue;
    const char *a = t.keys[i].key;
    const char *b = key;
    while (*a && *a == *b) {
      a++;
      b++;
    }
    if (*a == 0 && *b == 0) return i;
  }
  return -1;
}

// CRotationMatrix::SetRotation2(deg * M_PI_180) (src/algebra.cpp:198-247,
// 296-302): from the identity, rotations about z, y and x by the vector's z,
// y and x angles multiplied onto the right, each skipped for a zero angle.
// out[0]: 1 when every angle is zero (RotateVector returns its argument),
// out[1..9]: the matrix, row-major.
inline void keyed_rotation(const double deg[3], double *out) {
  const double k = 0.01745329251994329576923690768489;  // M_PI_180 (fractal.h:45-46)
  double m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  bool zero = true;
  for (int axis = 2; axis >= 0; axis--) {
    const double a = deg[axis] * k;
    if (a == 0.0) continue;
    const double sn = std::sin(a), cs = std::cos(a);
    double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (axis == 0) { r[0] = 1.0; r[4] = cs; r[8] = cs; r[5] = -sn; r[7] = sn; }
    if (axis == 1) { r[4] = 1.0; r[8] = cs; r[0] = cs; r[6] = -sn; r[2] = sn; }
    if (axis == 2) { r[8] = 1.0; r[0] = cs; r[4] = cs; r[1] = -sn; r[3] = sn; }
    double t[9];
    for (int row = 0; row < 3; row++)
      for (int col = 0; col < 3; col++)
        t[row * 3 + col] = m[row * 3 + 0] * r[col] + m[row * 3 + 1] * r[3 + col] + m[row * 3 + 2] * r[6 + col];
    for (int j = 0; j < 9; j++) m[j] = t[j];
    zero = false;
  }
  out[0] = zero ? 1.0 : 0.0;
  for (int j = 0; j < 9; j++) out[1 + j] = m[j];
}

inline double named_field(const mbr_fractal &f, int id) {
  switch (id) {
    case NF_MB_LIMIT: return f.mandelbox_folding_limit;
    case NF_MB_VALUE: return f.mandelbox_folding_value;
    case NF_MB_SCALE: return f.mandelbox_scale;
    case NF_ADE_SCALE1: return f.analytic_de_scale1;
    case NF_ADE_OFFSET1: return f.analytic_de_offset1;
    case NF_MB_MIN_R: return f.mandelbox_folding_min_radius;
    case NF_MB_FIXED_R: return f.mandelbox_folding_fixed_radius;
    case NF_POWER: return f.bulb_power;
    case NF_ALPHA: return f.bulb_alpha_angle_offset * 0.01745329251994329576923690768489;
    case NF_BETA: return f.bulb_beta_angle_offset * 0.01745329251994329576923690768489;
    default: return f.transf_scale3;
  }
}

// One value into x[] as its kind stores it: an int truncated toward zero
// (as cParameterContainer::Set<int> of the double), a bool 0 / 1.
inline void put_keyed(const FormulaKey &k, const double *v, double *x) {
  switch (k.kind) {
    case PK_INT: x[k.x] = double(int(v[0])); break;
    case PK_BOOL: x[k.x] = v[0] != 0.0 ? 1.0 : 0.0; break;
    case PK_VEC3: x[k.x] = v[0]; x[k.x + 1] = v[1]; x[k.x + 2] = v[2]; break;
    case PK_ROT: keyed_rotation(v, x + k.x); break;
    default: x[k.x] = v[0]; break;
  }
}

// The parameter block of a keyed formula: every key's default (a NAMED
// entry's field), then the values f.param lists.  Returns -1 when the block is filled, else the index of the
// first entry of f.param that is malformed (a key without its NUL, one the
// formula does not read, a non-finite value or an int out of range); -2 when
// n_params is out of range.
inline int pack_keyed(const mbr_fractal &f, double *x) {
  for (int j = 0; j < MBR_SLOT_X; j++) x[j] = 0.0;
  const KeyTable t = formula_keys(f.formula);
  if (f.n_params < 0 || f.n_params > MBR_MAX_FORMULA_PARAMS) return -2;
  for (int i = 0; i < t.n; i++) {
    if (t.keys[i].kind == PK_NAMED) {
      x[t.keys[i].x] = named_field(f, int(t.keys[i].def[0]));
    } else if (t.keys[i].kind == PK_NAMED3) {  // mandelbox_offset, the one vector field
      for (int c = 0; c < 3; c++) x[t.keys[i].x + c] = f.mandelbox_offset[c];
    } else {
      put_keyed(t.keys[i], t.keys[i].def, x);
    }
  }
  for (int j = 0; j < f.n_params; j++) {
    const mbr_formula_param &q = f.param[j];
    bool terminated = false;
    for (int c = 0; c < MBR_PARAM_KEY_LEN; c++)
      if (q.key[c] == 0) terminated = true;
    if (!terminated) return j;
    const int i = find_key(t, q.key);
    if (i < 0) return j;
    const int nv = t.keys[i].kind == PK_VEC3 || t.keys[i].kind == PK_ROT ? 3 : 1;
    for (int c = 0; c < nv; c++)
      if (!std::isfinite(q.value[c])) return j;
    if (t.keys[i].kind == PK_INT && !(q.value[0] > -2147483648.0 && q.value[0] < 2147483648.0)) return j;
    put_keyed(t.keys[i], q.value, x);
  }
  if (f.formula == MBR_FORMULA_DIFS_HEXTGRID2) {  // its constants, computed on the host as the reference computes them
    x[HGX_COS6] = std::cos(3.14159265358979323846 / 6.0);
    x[HGX_SIN6] = std::sin(3.14159265358979323846 / 6.0);
  }
  if (f.formula == MBR_FORMULA_GENERALIZED_FOLD_BOX) {  // the derived part of its block
    x[GFX_MAIN_ON] = f.mandelbox_main_rotation_enabled ? 1.0 : 0.0;
    keyed_rotation(f.mandelbox_rotation_main, x + GFX_MAIN_ROT);
    x[GFX_SIDES] = generalized_fold_box_planes(int(x[GFX_TYPE]), x + GFX_NV);
  }
  return -1;
}
#endif

}  // namespace mbr
