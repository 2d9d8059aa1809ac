// fract_loader.cpp - a mandelbulber2 settings file (.fract text) read into
// the structs of this path: mbr_scene, mbr_camera, mbr_render_params.
//
// The reference loads settings in cSettings::LoadFromString and Decode
// (src/settings.cpp:513-527, 647-977), line by line in DecodeOneLine
// (:1015-1240), with version-dependent renames in Compatibility (:1262-1492)
// and Compatibility2 (:1494-1754), and then migrates files older than 2.35
// to its objects tree (MigrateToObjectsTree, :2551-2953).  All example
// scenes the reference ships are of that older, flat form:
//
//   # Mandelbulber settings file
//   # version 2.33
//   # only modified parameters            (or "all parameters")
//   [main_parameters]
//   name value;                           (comma or point decimals, vectors space-separated)
//   [fractal_1]
//   name value;
//
// This reader restates that flat form for the parameters the DE path reads:
// formulas and the hybrid sequence, the iteration and bailout settings,
// camera, raymarching quality, the main light, AO and the 8-bit conversion.
// Primitives joined by union (plane, box, sphere, water, torus, cylinder,
// circle, rectangle, cone, prism, ellipsoid) are read into mbr_scene.primitive, and so are the
// DE method and function (the delta DE included).  Geometry this path
// does not build (other formulas, boolean combinations, other primitives or
// operators, transforms) makes the call
// return MBR_EUNSUPPORTED with each item named in the report; shading
// parameters outside the path (materials, fog, glow, reflections, textures,
// further lights) are counted and listed as ignored.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mbr.h"
#include "formula_params.h"

namespace {

const int kSlots = MBR_MAX_FRACTALS;

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n' || s[a] == '\v' || s[a] == '\f')) a++;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n' || s[b - 1] == '\v' ||
                   s[b - 1] == '\f'))
    b--;
  return s.substr(a, b - a);
}

std::string strip_quotes(const std::string &s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return trim(s.substr(1, s.size() - 2));
  return s;
}

bool starts_with(const std::string &s, const char *p) { return s.compare(0, std::strlen(p), p) == 0; }

// One "name value;" line (DecodeOneLine, settings.cpp:1017-1043): the name
// ends at the first space, the value at the first semicolon; enclosing
// quotes are removed from both.  Whatever follows the semicolon (an
// animation script) is not read.
bool split_line(const std::string &line, std::string &name, std::string &value) {
  const size_t sp = line.find(' ');
  const size_t sc = line.find(';');
  if (sp == std::string::npos || sc == std::string::npos || sc <= sp) return false;
  name = strip_quotes(trim(line.substr(0, sp)));
  value = strip_quotes(trim(line.substr(sp + 1, sc - sp - 1)));
  return true;
}

// Numbers are written with the saving locale's decimal separator: a comma
// reads as a point (everyLocaleDouble, settings.cpp:2063-2073).
bool parse_double(const std::string &v, double &out) {
  std::string t = trim(v);
  for (char &c : t)
    if (c == ',') c = '.';
  if (t.empty()) return false;
  char *end = nullptr;
  const double d = std::strtod(t.c_str(), &end);
  if (end == t.c_str() || *end != '\0') return false;
  out = d;
  return true;
}

bool parse_int(const std::string &v, int &out) {
  double d;
  if (!parse_double(v, d) || d != std::floor(d) || std::fabs(d) > 2147483647.0) return false;
  out = int(d);
  return true;
}

bool parse_bool(const std::string &v, int &out) {
  const std::string t = trim(v);
  if (t == "true" || t == "1") out = 1;
  else if (t == "false" || t == "0") out = 0;
  else return false;
  return true;
}

bool parse_vec3(const std::string &v, double out[3]) {
  std::vector<std::string> parts;
  std::string cur;
  for (char c : v) {
    if (c == ' ' || c == '\t') {
      if (!cur.empty()) parts.push_back(cur);
      cur.clear();
    } else {
      cur += c;
    }
  }
  if (!cur.empty()) parts.push_back(cur);
  if (parts.size() != 3) return false;
  for (int i = 0; i < 3; i++)
    if (!parse_double(parts[i], out[i])) return false;
  return true;
}

// "name_K" with K in 1..9: the base name and the 0-based slot.
bool indexed(const std::string &name, std::string &base, int &slot) {
  const size_t u = name.rfind('_');
  if (u == std::string::npos || u + 1 >= name.size()) return false;
  int k = 0;
  for (size_t i = u + 1; i < name.size(); i++) {
    if (name[i] < '0' || name[i] > '9') return false;
    k = k * 10 + (name[i] - '0');
    if (k > 99) return false;
  }
  if (k < 1 || k > kSlots) return false;
  base = name.substr(0, u);
  slot = k - 1;
  return true;
}

struct V3 {
  double x, y, z;
};
V3 v3(const double a[3]) { return V3{a[0], a[1], a[2]}; }
V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 mul(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double length(V3 a) { return std::sqrt(dot(a, a)); }
V3 normalize(V3 a) {
  const double l = length(a);
  return l > 0.0 ? mul(a, 1.0 / l) : a;
}
// Rodrigues' rotation of v about the unit axis a (CVector3::RotateAroundVectorByAngle, algebra.cpp:71-77)
V3 rotate_about(V3 v, V3 a, double angle) {
  V3 r = mul(v, std::cos(angle));
  r = add(r, mul(cross(a, v), std::sin(angle)));
  return add(r, mul(a, dot(a, v) * (1.0 - std::cos(angle))));
}
// atan2 angles of CVector3::GetAlpha / GetBeta (algebra.hpp)
double get_alpha(V3 v) { return std::atan2(v.y, v.x); }
double get_beta(V3 v) { return std::atan2(v.z, std::sqrt(v.x * v.x + v.y * v.y)); }

// The camera frame of cCameraTarget::SetCameraTargetTop (camera_target.cpp:88-126).
void camera_frame(V3 camera, V3 target, V3 top_in, V3 &forward, V3 &top, V3 &right) {
  const bool same = camera.x == target.x && camera.y == target.y && camera.z == target.z;
  forward = normalize(same ? V3{0.0, 1.0, 0.0} : sub(target, camera));
  const double yaw = get_alpha(forward) - 0.5 * M_PI;
  const double pitch = get_beta(forward);
  V3 t = normalize(top_in);
  t = rotate_about(t, V3{0.0, 0.0, 1.0}, -yaw);
  t = rotate_about(t, V3{1.0, 0.0, 0.0}, -pitch);
  const double roll = -std::atan2(t.z, t.x) + 0.5 * M_PI;
  // CorrectAngle only wraps into (-pi, pi]; the rotations below are periodic
  top = V3{0.0, 0.0, 1.0};
  top = rotate_about(top, V3{0.0, 1.0, 0.0}, roll);
  top = rotate_about(top, V3{1.0, 0.0, 0.0}, pitch);
  top = rotate_about(top, V3{0.0, 0.0, 1.0}, yaw);
  right = cross(forward, top);
}

// CRotationMatrix::SetRotation(CVector3) = RotateZ(x) RotateX(y) RotateY(z) applied to v
// (algebra.cpp:265-271; RotateZ/X/Y post-multiply the matrix by the axis rotation).
V3 rotate_zxy(V3 v, V3 angles) {
  // M = Rz(a) * Rx(b) * Ry(c); M v = Rz(a) (Rx(b) (Ry(c) v))
  const double ca = std::cos(angles.x), sa = std::sin(angles.x);
  const double cb = std::cos(angles.y), sb = std::sin(angles.y);
  const double cc = std::cos(angles.z), sc = std::sin(angles.z);
  V3 r{cc * v.x + sc * v.z, v.y, -sc * v.x + cc * v.z};  // Ry(c)
  r = V3{r.x, cb * r.y - sb * r.z, sb * r.y + cb * r.z};  // Rx(b)
  return V3{ca * r.x - sa * r.y, sa * r.x + ca * r.y, r.z};  // Rz(a)
}

// A legacy primitive_<type>_<n>_* block (settings.cpp:1058-1080, initparameters.cpp:1313-1420)
struct PrimRead {
  std::string key;  // "<type>_<n>"
  int type = 0;     // mbr_primitive_type, 0: a kind not built here
  std::string type_name;
  int enabled = 0;  // InitPrimitiveParams: "_enabled" false
  int boolean_operator = 1;  // primBooleanOperatorOR
  int smooth = 0;
  mbr_primitive q;
};

struct Reader {
  double version = 0.0;
  std::vector<PrimRead> prims;
  int frame_no = 0;
  std::vector<std::string> unsupported, ignored, notes, errors;

  // main parameters (defaults: initparameters.cpp)
  int N = 250;
  int hybrid = 0, boolean_ops = 0;
  int formula[kSlots];
  int slot_enable[kSlots];
  // formula transforms (formula_position/_rotation/_scale/_repeat of each
  // slot) and the legacy global fractal transform (fractal_position,
  // fractal_rotation, repeat; MigrateLegacyParamsToFractal,
  // settings.cpp:2372-2401, copies a non-default one into every slot)
  double f_pos[kSlots][3] = {}, f_rot[kSlots][3] = {}, f_rep[kSlots][3] = {}, f_scale[kSlots];
  double g_pos[3] = {0, 0, 0}, g_rot[3] = {0, 0, 0}, g_rep[3] = {0, 0, 0};
  // the per-fractal node parameters of a boolean combination (the fractal
  // containers' julia_mode, julia_c, fractal_constant_factor, initial_waxis,
  // formula_maxiter; initparameters.cpp:705-715) and boolean_operator_K
  int f_julia[kSlots] = {}, f_maxiter[kSlots], bool_op[kSlots + 1], bool_op_set[kSlots + 1] = {};
  double f_julia_c[kSlots][3] = {}, f_cmul[kSlots][3], f_w0[kSlots] = {};
  int ao_enabled = 0, ao_mode = 2;
  double ao_intensity = 1.0;
  int ao_quality = 4;
  double ao_fast_tune = 1.0;
  // light 1 (initparameters.cpp:1895-1950)
  int light_enabled = 1, light_shadows = 1, light_penetrating = 1, light_relative = 1, light_use_target = 0;
  int light_type = 0;  // 0 directional
  int light_defined = 0;
  double light_rot[3] = {-45.0, 45.0, 0.0};
  double light_alpha = -45.0, light_beta = 45.0;
  double light_soft_cone = 1.0, light_intensity = 1.0, all_lights_intensity = 1.0;
  double light_pos[3] = {0.0, 0.0, 0.0}, light_target[3] = {0.0, 0.0, 0.0};

  Reader() {
    for (int i = 0; i < kSlots; i++) {
      formula[i] = i == 0 ? MBR_FORMULA_MANDELBULB : MBR_FORMULA_NONE;
      slot_enable[i] = 1;
      f_scale[i] = 1.0;
      f_maxiter[i] = 250;
      for (int k = 0; k < 3; k++) f_cmul[i][k] = 1.0;
    }
  }

  void bad(const std::string &name, const std::string &value) { errors.push_back(name + " '" + value + "'"); }
};

// Renames of older files that reach the keys read here (Compatibility,
// settings.cpp:1283-1466).
void compatibility(const Reader &R, std::string &name, std::string &value) {
  const double v = R.version;
  if (v <= 2.04 && name == "fractal_constant_factor") {
    const std::string t = trim(value);
    if (t.find(' ') == std::string::npos) value = t + " " + t + " " + t;
  }
  if (v <= 2.06 && name == "linear_DE_mode") {
    name = "delta_DE_function";
    value = "1";
  }
  if (v < 2.09 && name == "delta_DE_function") {
    if (value == "0") value = "2";
    else if (value == "2") value = "0";
  }
  if (v < 2.25) {
    struct Ren {
      const char *from, *to;
    };
    static const Ren ren[] = {{"main_light_intensity", "light1_intensity"},
                              {"main_light_alpha", "light1_alpha"},
                              {"main_light_beta", "light1_beta"},
                              {"penetrating_lights", "light1_penetrating"},
                              {"shadows_enabled", "light1_cast_shadows"},
                              {"shadows_cone_angle", "light1_soft_shadow_cone"},
                              {"main_light_enable", "light1_enabled"},
                              {"main_light_position_relative", "light1_relative_position"}};
    for (const Ren &r : ren)
      if (name == r.from) name = r.to;
  }
}

// primitive_<type>_<n>_<param> (the legacy flat form; cPrimitives::PrimitiveNameToEnum)
void read_primitive_param(Reader &R, const std::string &full, const std::string &value) {
  const std::string rest = full.substr(10);  // after "primitive_"
  const size_t u1 = rest.find('_');
  const size_t u2 = (u1 == std::string::npos) ? u1 : rest.find('_', u1 + 1);
  int index = 0;
  if (u2 == std::string::npos || !parse_int(rest.substr(u1 + 1, u2 - u1 - 1), index)) {
    R.unsupported.push_back(full + " (primitive parameter)");
    return;
  }
  const std::string tname = rest.substr(0, u1), key = rest.substr(0, u2);
  std::string param = rest.substr(u2 + 1);
  // settings.cpp:1365-1372: before 2.13 the water's "amplitude" is its relative amplitude
  if (R.version < 2.13 && tname == "water" && param == "amplitude") param = "relative_amplitude";
  PrimRead *pr = nullptr;
  for (PrimRead &x : R.prims)
    if (x.key == key) pr = &x;
  if (!pr) {
    static const struct {
      const char *name;
      int type;
    } kinds[] = {{"plane", MBR_PRIMITIVE_PLANE},       {"box", MBR_PRIMITIVE_BOX},
                 {"sphere", MBR_PRIMITIVE_SPHERE},     {"water", MBR_PRIMITIVE_WATER},
                 {"torus", MBR_PRIMITIVE_TORUS},       {"cylinder", MBR_PRIMITIVE_CYLINDER},
                 {"circle", MBR_PRIMITIVE_CIRCLE},     {"rectangle", MBR_PRIMITIVE_RECTANGLE},
                 {"cone", MBR_PRIMITIVE_CONE},         {"prism", MBR_PRIMITIVE_PRISM},
                 {"ellipsoid", MBR_PRIMITIVE_ELLIPSOID}};
    int type = -1;
    for (const auto &k : kinds)
      if (tname == k.name) type = k.type;
    if (type < 0) {
      R.unsupported.push_back(full + " (unknown primitive)");
      return;
    }
    R.prims.push_back(PrimRead());
    pr = &R.prims.back();
    pr->key = key;
    pr->type = type;
    pr->type_name = tname;
    mbr_primitive_defaults(&pr->q, type);
  }
  mbr_primitive &q = pr->q;
  double d;
  int b;
  double v[3];
  auto vec = [&](double *dst) {
    if (parse_vec3(value, v)) std::memcpy(dst, v, sizeof(v)); else R.bad(full, value);
  };
  auto num = [&](double &dst) {
    if (parse_double(value, d)) dst = d; else R.bad(full, value);
  };
  auto flag = [&](int32_t &dst) {
    if (parse_bool(value, b)) dst = b; else R.bad(full, value);
  };
  if (param == "enabled") {
    if (parse_bool(value, b)) pr->enabled = b; else R.bad(full, value);
  } else if (param == "position") vec(q.position);
  else if (param == "rotation") vec(q.rotation);
  else if (param == "repeat") vec(q.repeat);
  else if (param == "size") vec(q.size);
  else if (param == "limits_min") vec(q.limits_min);
  else if (param == "limits_max") vec(q.limits_max);
  else if (param == "scale") num(q.scale);
  else if (param == "radius") num(q.radius);
  else if (param == "height") num(q.height);
  else if (param == "width") num(q.width);
  else if (param == "tube_radius") num(q.tube_radius);
  else if (param == "radius_lpow") num(q.radius_lpow);
  else if (param == "tube_radius_lpow") num(q.tube_radius_lpow);
  else if (param == "rounding") num(q.rounding);
  else if (param == "wall_thickness") num(q.wall_thickness);
  else if (param == "relative_amplitude") num(q.relative_amplitude);
  else if (param == "length") num(q.length);
  else if (param == "anim_speed") num(q.anim_speed);
  else if (param == "anim_progression_speed") num(q.anim_progression_speed);
  else if (param == "prism_angle") num(q.prism_angle);
  else if (param == "trangle_height") num(q.triangle_height);  // the reference's key
  else if (param == "empty") flag(q.empty);
  else if (param == "limits_enable") flag(q.limits_enable);
  else if (param == "caps") flag(q.caps);
  else if (param == "iterations") {
    if (parse_int(value, b)) q.iterations = b; else R.bad(full, value);
  } else if (param == "boolean_operator") {
    if (parse_int(value, b)) pr->boolean_operator = b; else R.bad(full, value);
  } else if (param == "smooth_de_combine_enable") {
    if (parse_bool(value, b)) pr->smooth = b; else R.bad(full, value);
  } else if (param == "wave_from_objects_enable" || param == "wave_from_objects_relative_amplitude") {
    // the water's distance from other objects is 1e20 in the objects-tree walk
    // (calculate_distance.cpp:385-396): the wave from objects has no effect
    R.ignored.push_back(full);
  } else {
    // material, colour, reflection, name, object id, calculation order,
    // smooth-combine distance: shading or tree bookkeeping
    R.ignored.push_back(full);
  }
}

// A fractal container's node parameter (julia_mode, julia_c,
// fractal_constant_factor, initial_waxis, formula_maxiter) of slot `slot`:
// true when `base` is one of them.
bool read_node_param(Reader &R, int slot, const std::string &base, const std::string &value) {
  int b;
  double d, v[3];
  if (base == "julia_mode") {
    if (parse_bool(value, b)) R.f_julia[slot] = b; else R.bad(base, value);
  } else if (base == "julia_c") {
    if (parse_vec3(value, v)) std::memcpy(R.f_julia_c[slot], v, sizeof(v)); else R.bad(base, value);
  } else if (base == "fractal_constant_factor") {
    if (parse_vec3(value, v)) std::memcpy(R.f_cmul[slot], v, sizeof(v)); else R.bad(base, value);
  } else if (base == "initial_waxis") {
    if (parse_double(value, d)) R.f_w0[slot] = d; else R.bad(base, value);
  } else if (base == "formula_maxiter") {
    if (parse_int(value, b)) R.f_maxiter[slot] = b; else R.bad(base, value);
  } else {
    return false;
  }
  return true;
}

void read_fractal_param(Reader &R, mbr_scene *sc, int slot, const std::string &name, const std::string &value) {
  mbr_fractal &f = sc->fractal[slot];
  double d;
  int b;
  double v[3];
  if (name == "power") {
    if (parse_double(value, d)) f.bulb_power = d; else R.bad(name, value);
  } else if (name == "alpha_angle_offset") {
    if (parse_double(value, d)) f.bulb_alpha_angle_offset = d; else R.bad(name, value);
  } else if (name == "beta_angle_offset") {
    if (parse_double(value, d)) f.bulb_beta_angle_offset = d; else R.bad(name, value);
  } else if (name == "mandelbox_scale") {
    if (parse_double(value, d)) f.mandelbox_scale = d; else R.bad(name, value);
  } else if (name == "mandelbox_folding_limit") {
    if (parse_double(value, d)) f.mandelbox_folding_limit = d; else R.bad(name, value);
  } else if (name == "mandelbox_folding_value") {
    if (parse_double(value, d)) f.mandelbox_folding_value = d; else R.bad(name, value);
  } else if (name == "mandelbox_folding_min_radius") {
    if (parse_double(value, d)) f.mandelbox_folding_min_radius = d; else R.bad(name, value);
  } else if (name == "mandelbox_folding_fixed_radius") {
    if (parse_double(value, d)) f.mandelbox_folding_fixed_radius = d; else R.bad(name, value);
  } else if (name == "mandelbox_offset") {
    if (parse_vec3(value, v)) std::memcpy(f.mandelbox_offset, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "transf_scale_3") {
    if (parse_double(value, d)) f.transf_scale3 = d; else R.bad(name, value);
  } else if (name == "cadd") {  // Aexion (fractal.cpp:118)
    if (parse_double(value, d)) f.aexion_cadd = d; else R.bad(name, value);
  } else if (name == "analyticDE_enabled") {
    if (parse_bool(value, b)) f.analytic_de_enabled = b; else R.bad(name, value);
  } else if (name == "analyticDE_scale_1") {
    if (parse_double(value, d)) f.analytic_de_scale1 = d; else R.bad(name, value);
  } else if (name == "analyticDE_offset_1") {
    if (parse_double(value, d)) f.analytic_de_offset1 = d; else R.bad(name, value);
  } else if (name == "mandelbox_rotations_enabled") {
    if (parse_bool(value, b)) f.mandelbox_rotations_enabled = b; else R.bad(name, value);
  } else if (name == "mandelbox_main_rotation_enabled") {
    if (parse_bool(value, b)) f.mandelbox_main_rotation_enabled = b; else R.bad(name, value);
  } else if (name == "mandelbox_rotation_main") {
    if (parse_vec3(value, v)) std::memcpy(f.mandelbox_rotation_main, v, sizeof(v)); else R.bad(name, value);
  } else if ((starts_with(name, "mandelbox_rotation_neg_") || starts_with(name, "mandelbox_rotation_pos_")) &&
             name.size() == 24 && name[23] >= '1' && name[23] <= '3') {
    // rotation[0][k] = mandelbox_rotation_neg_(k+1), rotation[1][k] = ..._pos_(k+1) (fractal.cpp:69-73)
    double *dst = (name[19] == 'n' ? f.mandelbox_rotation_neg : f.mandelbox_rotation_pos)[name[23] - '1'];
    if (parse_vec3(value, v)) std::memcpy(dst, v, sizeof(v)); else R.bad(name, value);
  } else if (starts_with(name, "IFS_")) {  // kaleidoscopic IFS (initparameters.cpp:724-743)
    const std::string k = name.substr(4);
    // indexed vector parameters: IFS_direction_0 .. IFS_enabled_8
    int idx = -1;
    std::string base = k;
    const size_t u = k.rfind('_');
    if (u != std::string::npos && u + 2 == k.size() && k[u + 1] >= '0' && k[u + 1] <= '8') {
      idx = k[u + 1] - '0';
      base = k.substr(0, u);
    }
    if (idx >= 0 && base == "direction") {
      if (parse_vec3(value, v)) std::memcpy(f.ifs_direction[idx], v, sizeof(v)); else R.bad(name, value);
    } else if (idx >= 0 && base == "rotations") {
      if (parse_vec3(value, v)) std::memcpy(f.ifs_rotations[idx], v, sizeof(v)); else R.bad(name, value);
    } else if (idx >= 0 && base == "distance") {
      if (parse_double(value, d)) f.ifs_distance[idx] = d; else R.bad(name, value);
    } else if (idx >= 0 && base == "intensity") {
      if (parse_double(value, d)) f.ifs_intensity[idx] = d; else R.bad(name, value);
    } else if (idx >= 0 && base == "enabled") {
      if (parse_bool(value, b)) f.ifs_enabled[idx] = b; else R.bad(name, value);
    } else if (k == "scale") {
      if (parse_double(value, d)) f.ifs_scale = d; else R.bad(name, value);
    } else if (k == "rotation") {
      if (parse_vec3(value, v)) std::memcpy(f.ifs_rotation, v, sizeof(v)); else R.bad(name, value);
    } else if (k == "rotation_enabled") {
      if (parse_bool(value, b)) f.ifs_rotation_enabled = b; else R.bad(name, value);
    } else if (k == "offset") {
      if (parse_vec3(value, v)) std::memcpy(f.ifs_offset, v, sizeof(v)); else R.bad(name, value);
    } else if (k == "edge") {
      if (parse_vec3(value, v)) std::memcpy(f.ifs_edge, v, sizeof(v)); else R.bad(name, value);
    } else if (k == "edge_enabled") {
      if (parse_bool(value, b)) f.ifs_edge_enabled = b; else R.bad(name, value);
    } else if (k == "abs_x") {
      if (parse_bool(value, b)) f.ifs_abs_x = b; else R.bad(name, value);
    } else if (k == "abs_y") {
      if (parse_bool(value, b)) f.ifs_abs_y = b; else R.bad(name, value);
    } else if (k == "abs_z") {
      if (parse_bool(value, b)) f.ifs_abs_z = b; else R.bad(name, value);
    } else if (k == "menger_sponge_mode") {
      if (parse_bool(value, b)) f.ifs_menger_sponge_mode = b; else R.bad(name, value);
    } else {
      R.ignored.push_back("fractal_" + std::to_string(slot + 1) + "." + name);
    }
  } else if (name == "formula_iterations") {
    if (parse_int(value, b)) f.formula_iterations = b; else R.bad(name, value);
  } else if (name == "formula_weight") {
    if (parse_double(value, d)) f.formula_weight = d; else R.bad(name, value);
  } else if (name == "formula_start_iteration") {
    if (parse_int(value, b)) f.formula_start_iteration = b; else R.bad(name, value);
  } else if (name == "formula_stop_iteration") {
    if (parse_int(value, b)) f.formula_stop_iteration = b; else R.bad(name, value);
  } else if (read_node_param(R, slot, name, value)) {
    // a node parameter of the fractal container
  } else {
    // a parameter the slot's formula reads by key (formula_params.h)
    const mbr::KeyTable t = mbr::formula_keys(R.formula[slot]);
    const int k = mbr::find_key(t, name.c_str());
    if (k < 0) {
      R.ignored.push_back("fractal_" + std::to_string(slot + 1) + "." + name);
      return;
    }
    double val[3] = {0.0, 0.0, 0.0};
    bool ok;
    switch (t.keys[k].kind) {
      case mbr::PK_INT: ok = parse_int(value, b); val[0] = b; break;
      case mbr::PK_BOOL: ok = parse_bool(value, b); val[0] = b; break;
      case mbr::PK_VEC3:
      case mbr::PK_ROT: ok = parse_vec3(value, val); break;
      default: ok = parse_double(value, val[0]); break;
    }
    if (!ok) {
      R.bad(name, value);
      return;
    }
    int j = 0;
    while (j < f.n_params && std::strcmp(f.param[j].key, name.c_str()) != 0) j++;
    if (j == f.n_params) {
      if (f.n_params == MBR_MAX_FORMULA_PARAMS) {
        R.unsupported.push_back("fractal_" + std::to_string(slot + 1) + "." + name + " (more than " +
                                std::to_string(MBR_MAX_FORMULA_PARAMS) + " formula parameters)");
        return;
      }
      std::snprintf(f.param[j].key, MBR_PARAM_KEY_LEN, "%s", name.c_str());
      f.n_params++;
    }
    std::memcpy(f.param[j].value, val, sizeof(val));
  }
}

bool nonzero3(const double v[3]) { return v[0] != 0.0 || v[1] != 0.0 || v[2] != 0.0; }

// A node of an explicit objects tree with InitNodeParams' defaults
// (initparameters.cpp:2102-2125).
mbr_node tree_node(int type, int level, int index) {
  mbr_node n;
  std::memset(&n, 0, sizeof(n));
  n.type = type;
  n.level = level;
  n.index = index;
  n.enabled = 1;
  n.scale = 1.0;
  n.detail_level_multiplier = 1.0;
  n.smooth_combine_distance = 0.1;
  n.formula_maxiter = 250;
  for (int k = 0; k < 3; k++) n.fractal_constant_factor[k] = 1.0;
  return n;
}

// The legacy boolean mode (MigrateToObjectsTree, settings.cpp:2608-2712): the
// m slots with a formula combine left to right, ((f1 op f2) op f3) ..., each
// operator a group (boolean_operator_K: 0 intersection, 2 subtraction, else
// union; a missing one takes boolean_operator_1's value, else union), each
// fractal a node with its slot's formula transform (CopyFormulaTransform) and
// node parameters (CopyOneFractalParams; formula_maxiter is N for files
// before 2.29, settings.cpp:1721-1733), disabled when its fractal_enable_K is
// false.  The file's primitives join by union at the root.
void build_boolean_tree(Reader &R, mbr_scene *scene) {
  int en[kSlots], m = 0;
  for (int i = 0; i < kSlots; i++)
    if (R.formula[i] != MBR_FORMULA_NONE) en[m++] = i;
  if (m == 0) return;
  const int npr = scene->n_primitives;
  const int root_shift = npr > 0 ? 1 : 0;
  const int count = (2 * m - 1) + root_shift + npr;
  if (count > MBR_MAX_NODES || (m - 1) + root_shift > 8) {
    R.unsupported.push_back("boolean_operators with " + std::to_string(m) + " fractals and " + std::to_string(npr) +
                            " primitives (more than " + std::to_string(MBR_MAX_NODES) + " tree nodes)");
    return;
  }
  const int default_op = R.bool_op_set[1] ? R.bool_op[1] : 1;
  auto op_type = [&](int j) {  // the group joining fractals 0..j-1 with fractal j (ToNodeType, :2418-2426)
    int idx = en[j];
    if (idx < 1) idx = 1;
    const int op = R.bool_op_set[idx] ? R.bool_op[idx] : default_op;
    return op == 0 ? MBR_NODE_BOOLEAN_MUL : (op == 2 ? MBR_NODE_BOOLEAN_SUB : MBR_NODE_BOOLEAN_ADD);
  };
  auto fractal_node = [&](int j, int level) {
    const int k = en[j];
    mbr_node n = tree_node(MBR_NODE_FRACTAL, level, k);
    n.enabled = R.slot_enable[k] ? 1 : 0;
    std::memcpy(n.position, R.f_pos[k], sizeof(n.position));
    std::memcpy(n.rotation, R.f_rot[k], sizeof(n.rotation));
    std::memcpy(n.repeat, R.f_rep[k], sizeof(n.repeat));
    n.scale = R.f_scale[k];
    n.formula_maxiter = R.version < 2.29 ? R.N : R.f_maxiter[k];
    n.julia_mode = R.f_julia[k];
    std::memcpy(n.julia_c, R.f_julia_c[k], sizeof(n.julia_c));
    std::memcpy(n.fractal_constant_factor, R.f_cmul[k], sizeof(n.fractal_constant_factor));
    n.initial_waxis = R.f_w0[k];
    return n;
  };
  int nn = 0;
  if (root_shift) scene->node[nn++] = tree_node(MBR_NODE_BOOLEAN_ADD, 0, 0);
  if (m == 1) {
    scene->node[nn++] = fractal_node(0, root_shift);
  } else {
    // preorder: the groups from the root inward, then fractals 0 and 1 in
    // the innermost group, then fractal j in the group that joins it
    for (int j = m - 1; j >= 1; j--) scene->node[nn++] = tree_node(op_type(j), root_shift + (m - 1 - j), 0);
    scene->node[nn++] = fractal_node(0, root_shift + m - 1);
    scene->node[nn++] = fractal_node(1, root_shift + m - 1);
    for (int j = 2; j < m; j++) scene->node[nn++] = fractal_node(j, root_shift + m - j);
  }
  for (int k = 0; k < npr; k++) scene->node[nn++] = tree_node(MBR_NODE_PRIMITIVE, 1, k);
  scene->n_nodes = nn;
}

void read_main_param(Reader &R, mbr_scene *sc, mbr_camera *cam, mbr_render_params *p, std::string name,
                     std::string value) {
  compatibility(R, name, value);
  double d;
  int b;
  double v[3];
  std::string base;
  int slot;
  // per-slot parameters of the flat form: formula_K, formula_iterations_K, ...
  if (indexed(name, base, slot)) {
    mbr_fractal &f = sc->fractal[slot];
    if (base == "formula") {
      if (parse_int(value, b)) R.formula[slot] = b; else R.bad(name, value);
      return;
    }
    if (base == "formula_iterations") {
      if (parse_int(value, b)) f.formula_iterations = b; else R.bad(name, value);
      return;
    }
    if (base == "formula_weight") {
      if (parse_double(value, d)) f.formula_weight = d; else R.bad(name, value);
      return;
    }
    if (base == "formula_start_iteration") {
      if (parse_int(value, b)) f.formula_start_iteration = b; else R.bad(name, value);
      return;
    }
    if (base == "formula_stop_iteration") {
      if (parse_int(value, b)) f.formula_stop_iteration = b; else R.bad(name, value);
      return;
    }
    if (base == "dont_add_c_constant") {
      if (parse_bool(value, b)) f.dont_add_c_constant = b; else R.bad(name, value);
      return;
    }
    if (base == "check_for_bailout") {
      if (parse_bool(value, b)) f.check_for_bailout = b; else R.bad(name, value);
      return;
    }
    if (base == "fractal_enable") {
      if (parse_bool(value, b)) R.slot_enable[slot] = b; else R.bad(name, value);
      return;
    }
    if (base == "formula_position" || base == "formula_rotation" || base == "formula_repeat") {
      double *dst = base == "formula_position" ? R.f_pos[slot] : (base == "formula_rotation" ? R.f_rot[slot] : R.f_rep[slot]);
      if (parse_vec3(value, v)) std::memcpy(dst, v, sizeof(v)); else R.bad(name, value);
      return;
    }
    if (base == "formula_scale") {
      if (parse_double(value, d)) R.f_scale[slot] = d; else R.bad(name, value);
      return;
    }
    // julia_mode_K, julia_c_K, fractal_constant_factor_K, initial_waxis_K,
    // formula_maxiter_K, boolean_operator_K: read by the boolean combination only
    if (read_node_param(R, slot, base, value)) return;
    if (base == "boolean_operator") {
      if (parse_int(value, b)) {
        R.bool_op[slot + 1] = b;
        R.bool_op_set[slot + 1] = 1;
      } else {
        R.bad(name, value);
      }
      return;
    }
    if (base == "formula_material_id") {
      R.ignored.push_back(name);
      return;
    }
  }
  if (starts_with(name, "primitive_")) {
    read_primitive_param(R, name, value);
    return;
  }
  if (name == "frame_no") {
    if (!parse_int(value, b)) R.bad(name, value); else R.frame_no = b;
    return;
  }
  if (starts_with(name, "node_")) {
    R.unsupported.push_back(name + " (objects tree)");
    return;
  }
  // formula and sequence
  if (name == "N") {
    if (parse_int(value, b)) R.N = b; else R.bad(name, value);
  } else if (name == "minN") {
    if (parse_int(value, b)) sc->min_n = b; else R.bad(name, value);
  } else if (name == "bailout") {
    if (parse_double(value, d)) sc->bailout = d; else R.bad(name, value);
  } else if (name == "use_default_bailout") {
    if (parse_bool(value, b)) sc->use_default_bailout = b; else R.bad(name, value);
  } else if (name == "repeat_from") {
    if (parse_int(value, b)) sc->repeat_from = b; else R.bad(name, value);
  } else if (name == "hybrid_fractal_enable") {
    if (parse_bool(value, b)) R.hybrid = b; else R.bad(name, value);
  } else if (name == "boolean_operators") {
    if (parse_bool(value, b)) R.boolean_ops = b; else R.bad(name, value);
  } else if (name == "julia_mode") {
    if (parse_bool(value, b)) sc->julia_mode = b; else R.bad(name, value);
  } else if (name == "julia_c") {
    if (parse_vec3(value, v)) std::memcpy(sc->julia_c, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "fractal_constant_factor") {
    if (parse_vec3(value, v)) std::memcpy(sc->fractal_constant_factor, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "initial_waxis") {
    if (parse_double(value, d)) sc->initial_waxis = d; else R.bad(name, value);
  } else if (name == "linear_DE_offset") {
    if (parse_double(value, d)) sc->linear_de_offset = d; else R.bad(name, value);
  } else if (name == "delta_DE_function") {
    // 0 preferred, 1 linear, 2 logarithmic, 3 pseudo-Kleinian, 4 Jos Kleinian, 5 custom, 6 max axis
    if (parse_int(value, b) && b >= 0 && b <= 6) sc->delta_de_function = b;
    else R.bad(name, value);
  } else if (name == "delta_DE_method") {
    // 0 preferred (analytic for every formula built here), 1 forced delta, 2 forced analytic
    if (parse_int(value, b) && b >= 0 && b <= 2) sc->delta_de_method = b;
    else R.bad(name, value);
  } else if (name == "deltade_relative_delta") {
    if (parse_double(value, d) && d > 0.0 && std::isfinite(d)) sc->deltade_relative_delta = d;
    else R.bad(name, value);
  } else if (name == "iteration_threshold_mode") {
    if (parse_bool(value, b)) sc->iteration_threshold_mode = b; else R.bad(name, value);
  } else if (name == "interior_mode") {
    if (parse_bool(value, b)) sc->interior_mode = b; else R.bad(name, value);
  } else if (name == "all_primitives_position" || name == "all_primitives_rotation") {
    // the transform of the group that holds the primitives (settings.cpp:3113-3117)
    if (parse_vec3(value, v) && nonzero3(v)) R.unsupported.push_back(name + " (primitive group transform)");
  } else if (name == "fractal_position" || name == "fractal_rotation" || name == "repeat") {
    double *dst = name == "fractal_position" ? R.g_pos : (name == "fractal_rotation" ? R.g_rot : R.g_rep);
    if (parse_vec3(value, v)) std::memcpy(dst, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "formula_code") {
    R.unsupported.push_back(name + " (custom formula code)");
  // camera and image
  } else if (name == "camera") {
    if (parse_vec3(value, v)) std::memcpy(cam->camera, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "target") {
    if (parse_vec3(value, v)) std::memcpy(cam->target, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "camera_top") {
    if (parse_vec3(value, v)) std::memcpy(cam->top, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "fov") {
    if (parse_double(value, d)) cam->fov_deg = d; else R.bad(name, value);
  } else if (name == "image_width") {
    if (parse_int(value, b)) cam->width = b; else R.bad(name, value);
  } else if (name == "image_height") {
    if (parse_int(value, b)) cam->height = b; else R.bad(name, value);
  } else if (name == "perspective_type") {  // enumeration names of initparameters.cpp:121-122
    if (value == "three_point" || value == "0") cam->perspective_type = MBR_PROJECTION_THREE_POINT;
    else if (value == "fish_eye" || value == "1") cam->perspective_type = MBR_PROJECTION_FISH_EYE;
    else if (value == "equirectangular" || value == "2") cam->perspective_type = MBR_PROJECTION_EQUIRECTANGULAR;
    else if (value == "fish_eye_cut" || value == "3") cam->perspective_type = MBR_PROJECTION_FISH_EYE_CUT;
    else R.bad(name, value);
  } else if (name == "legacy_coordinate_system") {
    if (parse_bool(value, b)) cam->legacy_coordinate_system = b; else R.bad(name, value);
  } else if (name == "camera_rotation" || name == "camera_distance_to_target") {
    // derived from camera, target and top by the reference itself
  // raymarching quality
  } else if (name == "detail_level") {
    if (parse_double(value, d)) p->detail_level = d; else R.bad(name, value);
  } else if (name == "DE_factor") {
    if (parse_double(value, d)) p->de_factor = d; else R.bad(name, value);
  } else if (name == "view_distance_max") {
    if (parse_double(value, d)) p->view_distance_max = d; else R.bad(name, value);
  } else if (name == "smoothness") {
    if (parse_double(value, d)) p->smoothness = d; else R.bad(name, value);
  } else if (name == "max_raymarching_steps") {
    if (parse_int(value, b)) p->max_raymarching_steps = b; else R.bad(name, value);
  } else if (name == "advanced_quality") {  // CalcDistThresh clamps, RayMarching step limits
    if (parse_bool(value, b)) p->advanced_quality = b; else R.bad(name, value);
  } else if (name == "detail_size_min") {
    if (parse_double(value, d)) p->detail_size_min = d; else R.bad(name, value);
  } else if (name == "detail_size_max") {
    if (parse_double(value, d)) p->detail_size_max = d; else R.bad(name, value);
  } else if (name == "abs_min_marching_step") {
    if (parse_double(value, d)) p->abs_min_marching_step = d; else R.bad(name, value);
  } else if (name == "abs_max_marching_step") {
    if (parse_double(value, d)) p->abs_max_marching_step = d; else R.bad(name, value);
  } else if (name == "rel_min_marching_step") {
    if (parse_double(value, d)) p->rel_min_marching_step = d; else R.bad(name, value);
  } else if (name == "rel_max_marching_step") {
    if (parse_double(value, d)) p->rel_max_marching_step = d; else R.bad(name, value);
  } else if (name == "limits_enabled") {  // the limit box (calculate_distance.cpp:261-275)
    if (parse_bool(value, b)) sc->limits_enabled = b; else R.bad(name, value);
  } else if (name == "limit_min") {
    if (parse_vec3(value, v)) std::memcpy(sc->limit_min, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "limit_max") {
    if (parse_vec3(value, v)) std::memcpy(sc->limit_max, v, sizeof(v)); else R.bad(name, value);
  } else if (name == "box_folding") {  // the global folds (compute_fractal.cpp:190-202)
    if (parse_bool(value, b)) sc->box_folding = b; else R.bad(name, value);
  } else if (name == "box_folding_limit") {
    if (parse_double(value, d)) sc->box_folding_limit = d; else R.bad(name, value);
  } else if (name == "box_folding_value") {
    if (parse_double(value, d)) sc->box_folding_value = d; else R.bad(name, value);
  } else if (name == "spherical_folding") {
    if (parse_bool(value, b)) sc->spherical_folding = b; else R.bad(name, value);
  } else if (name == "spherical_folding_inner") {
    if (parse_double(value, d)) sc->spherical_folding_inner = d; else R.bad(name, value);
  } else if (name == "spherical_folding_outer") {
    if (parse_double(value, d)) sc->spherical_folding_outer = d; else R.bad(name, value);
  } else if (name == "slow_shading") {  // iteration-count normals (shader_calculate_normals.cpp:83-106)
    if (parse_bool(value, b)) p->slow_shading = b; else R.bad(name, value);
  } else if (name == "stereo_enabled") {
    // a switch that changes the image plane (stereo, render_worker.cpp:107-108,
    // 158-161, 268): refused when on
    if (!parse_bool(value, b)) R.bad(name, value);
    else if (b) R.unsupported.push_back(name + " true (stereo image)");
  } else if (name == "constant_DE_threshold") {
    if (parse_bool(value, b)) p->constant_de_threshold = b; else R.bad(name, value);
  } else if (name == "DE_thresh") {
    if (parse_double(value, d)) p->de_thresh = d; else R.bad(name, value);
  // 8-bit conversion (cImage::CalculatePixel)
  } else if (name == "brightness") {
    if (parse_double(value, d)) p->brightness = d; else R.bad(name, value);
  } else if (name == "contrast") {
    if (parse_double(value, d)) p->contrast = d; else R.bad(name, value);
  } else if (name == "gamma") {
    if (parse_double(value, d)) p->gamma = d; else R.bad(name, value);
  } else if (name == "saturation") {
    if (parse_double(value, d)) p->saturation = d; else R.bad(name, value);
  } else if (name == "hdr") {
    if (parse_bool(value, b)) p->hdr = b; else R.bad(name, value);
  // the main light
  } else if (starts_with(name, "light1_")) {
    R.light_defined = 1;
    const std::string k = name.substr(7);
    if (k == "enabled") {
      if (parse_bool(value, b)) R.light_enabled = b; else R.bad(name, value);
    } else if (k == "cast_shadows") {
      if (parse_bool(value, b)) R.light_shadows = b; else R.bad(name, value);
    } else if (k == "penetrating") {
      if (parse_bool(value, b)) R.light_penetrating = b; else R.bad(name, value);
    } else if (k == "relative_position") {
      if (parse_bool(value, b)) R.light_relative = b; else R.bad(name, value);
    } else if (k == "use_target_point") {
      if (parse_bool(value, b)) R.light_use_target = b; else R.bad(name, value);
    } else if (k == "type") {
      if (value == "directional" || value == "0") R.light_type = 0;
      else R.light_type = 1;
    } else if (k == "rotation") {
      if (parse_vec3(value, v)) std::memcpy(R.light_rot, v, sizeof(v)); else R.bad(name, value);
    } else if (k == "alpha") {
      if (parse_double(value, d)) R.light_alpha = d; else R.bad(name, value);
    } else if (k == "beta") {
      if (parse_double(value, d)) R.light_beta = d; else R.bad(name, value);
    } else if (k == "intensity") {
      if (parse_double(value, d)) R.light_intensity = d; else R.bad(name, value);
    } else if (k == "soft_shadow_cone") {
      if (parse_double(value, d)) R.light_soft_cone = d; else R.bad(name, value);
    } else if (k == "position") {
      if (parse_vec3(value, v)) std::memcpy(R.light_pos, v, sizeof(v)); else R.bad(name, value);
    } else if (k == "target") {
      if (parse_vec3(value, v)) std::memcpy(R.light_target, v, sizeof(v)); else R.bad(name, value);
    } else {
      R.ignored.push_back(name);
    }
  } else if (name == "all_lights_intensity") {  // multiplies every light's intensity (light.cpp:77-83)
    if (parse_double(value, d)) R.all_lights_intensity = d; else R.bad(name, value);
  } else if (name == "mat1_shading") {
    if (parse_double(value, d)) p->material_shading = d; else R.bad(name, value);
  // ambient occlusion
  } else if (name == "ambient_occlusion_enabled") {
    if (parse_bool(value, b)) R.ao_enabled = b; else R.bad(name, value);
  } else if (name == "ambient_occlusion_mode") {
    if (value == "fast") R.ao_mode = 0;
    else if (value == "multiple_rays") R.ao_mode = 1;
    else if (value == "screen_space") R.ao_mode = 2;
    else if (parse_int(value, b)) R.ao_mode = b;
    else R.bad(name, value);
  } else if (name == "ambient_occlusion_quality") {
    if (parse_int(value, b)) R.ao_quality = b; else R.bad(name, value);
  } else if (name == "ambient_occlusion_fast_tune") {
    if (parse_double(value, d)) R.ao_fast_tune = d; else R.bad(name, value);
  } else if (name == "ambient_occlusion") {
    if (parse_double(value, d)) R.ao_intensity = d; else R.bad(name, value);
  } else {
    R.ignored.push_back(name);
  }
}

void append(std::string &out, const std::string &s) {
  out += s;
  out += '\n';
}

}  // namespace

extern "C" mbr_status mbr_fract_parse(const char *text, mbr_scene *scene, mbr_camera *camera,
                                      mbr_render_params *params, char *report, int32_t report_size) {
  if (!text || !scene || !camera || !params) return MBR_EINVAL;
  Reader R;
  std::string rep;
  auto finish = [&](mbr_status st) {
    if (report && report_size > 0) {
      const size_t n = std::min(rep.size(), size_t(report_size - 1));
      std::memcpy(report, rep.data(), n);
      report[n] = '\0';
    }
    return st;
  };

  // lines split at \n, \r\n or \r of the trimmed text (settings.cpp:656-665)
  std::vector<std::string> lines;
  {
    const std::string all = trim(std::string(text));
    std::string cur;
    for (size_t i = 0; i < all.size(); i++) {
      const char c = all[i];
      if (c == '\r' || c == '\n') {
        lines.push_back(cur);
        cur.clear();
        if (c == '\r' && i + 1 < all.size() && all[i + 1] == '\n') i++;
      } else {
        cur += c;
      }
    }
    lines.push_back(cur);
  }
  // header (DecodeHeader, settings.cpp:540-601)
  if (lines.size() < 3) {
    append(rep, "error: not a Mandelbulber settings file (no header)");
    return finish(MBR_EINVAL);
  }
  if (lines[0].find("Mandelbulber settings file") == std::string::npos) {
    append(rep, "error: not a Mandelbulber settings file (wrong header)");
    return finish(MBR_EINVAL);
  }
  const size_t vp = lines[1].rfind("version");
  if (vp == std::string::npos || !parse_double(lines[1].substr(vp + 7), R.version)) {
    append(rep, "error: no version number in the header");
    return finish(MBR_EINVAL);
  }
  if (lines[2].find("all parameters") == std::string::npos &&
      lines[2].find("only modified parameters") == std::string::npos) {
    append(rep, "error: the header names no settings format (all / only modified parameters)");
    return finish(MBR_EINVAL);
  }

  // defaults (initparameters.cpp): scene and fractal slots, camera, quality, light 1
  mbr_scene_defaults(scene);
  mbr_camera_defaults(camera);
  mbr_render_params_defaults(params);
  const double top0[3] = {-0.1277753, 0.2555506, 0.958314};  // camera_top (initparameters.cpp:116)
  std::memcpy(camera->top, top0, sizeof(top0));
  params->ambient_intensity = 0.0;
  params->ao_rays = 0;

  std::string section;
  std::vector<std::pair<int, std::pair<std::string, std::string>>> fractal_lines;
  for (size_t l = 3; l < lines.size(); l++) {
    const std::string &line = lines[l];
    if (!line.empty() && line.front() == '[' && line.back() == ']') {  // CheckSection (settings.cpp:1247-1255)
      section = line.substr(1, line.size() - 2);
      continue;
    }
    if (section == "description" || section == "frames" || section == "keyframes") continue;
    const std::string t = trim(line);
    if (t.empty()) continue;
    std::string name, value;
    if (!split_line(t, name, value)) {
      if (section == "main_parameters" || starts_with(section, "fractal_")) R.errors.push_back("line " + std::to_string(l + 1) + ": '" + t + "'");
      continue;
    }
    if (section == "main_parameters") {
      read_main_param(R, scene, camera, params, name, value);
    } else if (starts_with(section, "fractal_")) {
      int k = 0;
      if (std::sscanf(section.c_str() + 8, "%d", &k) == 1 && k >= 1 && k <= kSlots)
        fractal_lines.push_back({k - 1, {name, value}});
      else
        R.ignored.push_back(section + "." + name);
    } else {
      R.ignored.push_back((section.empty() ? std::string("?") : section) + "." + name);
    }
  }
  for (const auto &fl : fractal_lines) read_fractal_param(R, scene, fl.first, fl.second.first, fl.second.second);

  if (!R.errors.empty()) {
    for (const std::string &e : R.errors) append(rep, "error: malformed value or line: " + e);
    return finish(MBR_EINVAL);
  }

  // formulas: a single fractal renders slot 1; a hybrid iterates every slot
  // whose formula is not none (MigrateToObjectsTree, settings.cpp:2716-2830)
  // a boolean combination of the slots with a formula (MigrateToObjectsTree,
  // settings.cpp:2608-2712) becomes an explicit objects tree (below)
  const bool boolean = R.boolean_ops && !R.hybrid;
  if (R.boolean_ops && R.hybrid) R.unsupported.push_back("boolean_operators with a hybrid (boolean combination of fractals)");
  scene->hybrid_fractal_enable = R.hybrid;
  int last = 0;
  for (int i = 0; i < kSlots; i++) {
    scene->fractal[i].formula = R.formula[i];
    if (R.formula[i] != MBR_FORMULA_NONE) last = i + 1;
  }
  scene->n_fractals = (R.hybrid || boolean) ? (last > 0 ? last : 1) : 1;
  // the scene holds one IFS block and one Mandelbox-rotation block
  int n_ifs = 0, n_box = 0;
  for (int i = 0; i < scene->n_fractals && (R.hybrid || boolean || i == 0); i++) {
    if (R.formula[i] == MBR_FORMULA_KALEIDOSCOPIC_IFS) n_ifs++;
    if (R.formula[i] == MBR_FORMULA_MANDELBOX) n_box++;
  }
  for (int i = 0; i < scene->n_fractals; i++) {
    const int f = R.formula[i];
    if (!R.hybrid && !boolean && i > 0) break;
    if (f == MBR_FORMULA_NONE) continue;
    if (f != MBR_FORMULA_MANDELBULB && f != MBR_FORMULA_MANDELBOX && f != MBR_FORMULA_MENGER_SPONGE &&
        f != MBR_FORMULA_MANDELBULB_POWER2 && f != MBR_FORMULA_HYPERCOMPLEX && f != MBR_FORMULA_KALEIDOSCOPIC_IFS &&
        f != MBR_FORMULA_XENODREAMBUIE && f != MBR_FORMULA_QUATERNION && f != MBR_FORMULA_AEXION &&
        mbr::formula_keys(f).n == 0)
      R.unsupported.push_back("formula_" + std::to_string(i + 1) + " " + std::to_string(f) +
                              " (formula not built here: 2 Mandelbulb, 3 Mandelbulb power 2, 4 hypercomplex, "
                              "5 quaternion, 7 Menger sponge, 8 Mandelbox, 10 kaleidoscopic IFS, 11 xenodreambuie, "
                              "16 box fold bulb pow 2, 19 aexion, 37 generalized fold box, 61 Menger mod 1, 103 pseudo-Kleinian, "
                              "101 pseudo-Kleinian std DE, 119 Abox mod 11, 125 box fold bulb pow 2 V2, 217 pseudo-Kleinian mod 4, "
                              "266 Mandelbulb Pupuku, 608 DIFS hextgrid2 are)");
    if (f == MBR_FORMULA_KALEIDOSCOPIC_IFS && n_ifs > 1)
      R.unsupported.push_back("formula_" + std::to_string(i + 1) + " 10 (kaleidoscopic IFS in more than one slot)");
    if (!R.slot_enable[i] && !boolean) R.unsupported.push_back("fractal_enable_" + std::to_string(i + 1) + " false");
    if (f == MBR_FORMULA_MANDELBOX && n_box > 1 &&
        (scene->fractal[i].mandelbox_rotations_enabled || scene->fractal[i].mandelbox_main_rotation_enabled))
      R.unsupported.push_back("fractal_" + std::to_string(i + 1) +
                              " rotations (Mandelbox rotations with more than one Mandelbox slot)");
  }
  if (!R.hybrid && R.formula[0] == MBR_FORMULA_NONE) R.unsupported.push_back("formula_1 0 (no fractal)");
  // enabled primitives join the fractal by union (MigrateToObjectsTree, settings.cpp:2866-2940)
  scene->n_primitives = 0;
  for (const PrimRead &pr : R.prims) {
    if (!pr.enabled) continue;
    const std::string nm = "primitive_" + pr.key;
    if (pr.boolean_operator != 1) {
      R.unsupported.push_back(nm + "_boolean_operator " + std::to_string(pr.boolean_operator) +
                              " (primitive combined other than by union)");
      continue;
    }
    if (pr.smooth) {
      R.unsupported.push_back(nm + "_smooth_de_combine_enable (smooth union)");
      continue;
    }
    if (pr.type == MBR_PRIMITIVE_WATER && pr.q.length == 0.0) {
      R.unsupported.push_back(nm + "_length 0 (water of zero wave length)");
      continue;
    }
    if (pr.type == MBR_PRIMITIVE_CONE && pr.q.height == 0.0) {
      R.unsupported.push_back(nm + "_height 0 (flat cone)");
      continue;
    }
    if (pr.type == MBR_PRIMITIVE_ELLIPSOID && !(pr.q.size[0] != 0.0 && pr.q.size[1] != 0.0 && pr.q.size[2] != 0.0)) {
      R.unsupported.push_back(nm + "_size with a zero axis");
      continue;
    }
    if (scene->n_primitives == MBR_MAX_PRIMITIVES) {
      R.unsupported.push_back(nm + " (more than " + std::to_string(MBR_MAX_PRIMITIVES) + " primitives)");
      continue;
    }
    if (pr.q.iterations < 0 || pr.q.iterations > 100) {
      R.unsupported.push_back(nm + "_iterations " + std::to_string(pr.q.iterations) + " (outside 0..100)");
      continue;
    }
    mbr_primitive q = pr.q;
    q.frame_no = R.frame_no;
    scene->primitive[scene->n_primitives++] = q;
  }
  // the node's iteration limit is the main N (CopyFractalParams, settings.cpp:2494-2501; the hybrid root :2775-2778)
  scene->formula_maxiter = R.N;

  // light 1 direction (cLight::Set, light.cpp:90-190): files before 2.25 give
  // alpha and beta; rotation is scaled by pi/180.8 as the reference does
  if (R.version < 2.25 && R.light_defined) {
    R.light_rot[0] = R.light_alpha;
    R.light_rot[1] = R.light_beta;
    R.light_rot[2] = 0.0;
  }
  params->shading_enable = R.light_enabled;
  params->shadow_enable = R.light_enabled && R.light_shadows;
  params->light_intensity = R.light_intensity * R.all_lights_intensity;
  if (R.light_type != 0) {
    append(rep, "note: light1 is not directional; the path lights with a directional light from its default rotation");
  }
  {
    V3 rot = mul(v3(R.light_rot), M_PI / 180.8);
    rot = V3{rot.x, -rot.y, rot.z};  // directional
    V3 dir;
    if (R.light_relative) {
      V3 fwd, top, right;
      camera_frame(v3(camera->camera), v3(camera->target), v3(camera->top), fwd, top, right);
      if (R.light_use_target && R.light_type == 0) {
        const V3 c = v3(camera->camera);
        const V3 dp = v3(R.light_pos), dt = v3(R.light_target);
        const V3 pos = add(c, add(add(mul(fwd, dp.z), mul(top, dp.y)), mul(right, dp.x)));
        const V3 tgt = add(c, add(add(mul(fwd, dt.z), mul(top, dt.y)), mul(right, dt.x)));
        dir = sub(pos, tgt);
        dir = length(dir) > 0.0 ? normalize(dir) : mul(fwd, -1.0);
      } else {
        dir = mul(fwd, -1.0);
        dir = rotate_about(dir, fwd, rot.z);
        dir = rotate_about(dir, right, rot.y);
        dir = rotate_about(dir, top, rot.x);
      }
    } else if (R.light_use_target && R.light_type == 0) {
      dir = sub(v3(R.light_pos), v3(R.light_target));
      dir = length(dir) > 0.0 ? normalize(dir) : V3{1.0, 0.0, 0.0};
    } else {
      dir = rotate_zxy(V3{0.0, -1.0, 0.0}, rot);
    }
    params->light_direction[0] = dir.x;
    params->light_direction[1] = dir.y;
    params->light_direction[2] = dir.z;
  }
  params->penetrating = R.light_penetrating;
  params->soft_shadow_cone = R.light_soft_cone;
  if (!(R.light_soft_cone >= 0.0 && R.light_soft_cone < 90.0)) {
    params->soft_shadow_cone = R.light_soft_cone < 0.0 ? 0.0 : 89.0;
    append(rep, "note: light1_soft_shadow_cone outside [0, 90) degrees: clamped");
  }

  // ambient occlusion: the multiple-rays mode maps onto 16 cosine-hemisphere
  // rays per hit, the fast mode onto its quality^2 - 1 samples along the
  // normal (quality and fast tune in the reference's ranges,
  // initparameters.cpp:215-216); the screen-space mode is not on this path
  if (R.ao_enabled) {
    if (R.ao_mode == 1) {
      params->ao_rays = 16;
      params->ambient_intensity = R.ao_intensity;
      append(rep, "note: ambient_occlusion (multiple rays): 16 cosine-hemisphere rays per hit");
    } else if (R.ao_mode == 0) {
      params->ao_fast = 1;
      params->ao_quality = std::min(10, std::max(1, R.ao_quality));
      params->ao_fast_tune = std::isfinite(R.ao_fast_tune) ? std::min(1e5, std::max(1e-5, R.ao_fast_tune)) : 1.0;
      params->ambient_intensity = R.ao_intensity;
    } else {
      append(rep, "note: ambient_occlusion mode screen space is not on this path; AO off");
    }
  }

  // the analytic Jos Kleinian DE function reads formula parameters not carried here
  if (scene->delta_de_function == MBR_DE_FUNCTION_JOS_KLEINIAN && scene->delta_de_method != MBR_DE_METHOD_FORCE_DELTA)
    R.unsupported.push_back("delta_DE_function 4 (the analytic Jos Kleinian DE function)");
  if (scene->delta_de_method == MBR_DE_METHOD_FORCE_DELTA)
    append(rep, "note: delta_DE_method 1 (forced delta DE): the plain FP64 engines render it");
  // the fractal's transform: a single fractal becomes the fractal node of
  // an explicit objects tree with the primitives beside it in the root union
  // (MigrateToObjectsTree with CopyFormulaTransform, settings.cpp:2471-2481,
  // 2713-2730, 2866-2940); hybrids and boolean combinations keep refusing it
  for (int i = 0; i < kSlots; i++) {
    for (int k = 0; k < 3; k++) {
      if (nonzero3(R.g_pos)) R.f_pos[i][k] = R.g_pos[k];
      if (nonzero3(R.g_rot)) R.f_rot[i][k] = R.g_rot[k];
      if (nonzero3(R.g_rep)) R.f_rep[i][k] = R.g_rep[k];
    }
  }
  const int iterated = R.hybrid ? scene->n_fractals : 1;
  bool transformed = false;
  for (int i = 0; i < iterated; i++)
    if (nonzero3(R.f_pos[i]) || nonzero3(R.f_rot[i]) || nonzero3(R.f_rep[i]) || R.f_scale[i] != 1.0) transformed = true;
  if (boolean) {
    build_boolean_tree(R, scene);
  } else if (transformed && (R.hybrid || R.boolean_ops)) {
    R.unsupported.push_back("formula or fractal transform of a hybrid or boolean combination");
  } else if (transformed) {
    if (!(std::fabs(R.f_scale[0]) > 1e-12)) {
      R.unsupported.push_back("formula_scale_1 0 (degenerate formula transform)");
    } else {
      mbr_node &n = scene->node[0];
      std::memset(&n, 0, sizeof(n));
      n.type = MBR_NODE_FRACTAL;
      n.index = 0;
      n.enabled = 1;
      std::memcpy(n.position, R.f_pos[0], sizeof(n.position));
      std::memcpy(n.rotation, R.f_rot[0], sizeof(n.rotation));
      std::memcpy(n.repeat, R.f_rep[0], sizeof(n.repeat));
      n.scale = R.f_scale[0];
      n.detail_level_multiplier = 1.0;
      n.smooth_combine_distance = 0.1;
      n.formula_maxiter = scene->formula_maxiter;
      n.julia_mode = scene->julia_mode;
      std::memcpy(n.julia_c, scene->julia_c, sizeof(n.julia_c));
      std::memcpy(n.fractal_constant_factor, scene->fractal_constant_factor, sizeof(n.fractal_constant_factor));
      n.initial_waxis = scene->initial_waxis;
      scene->n_nodes = 1;
      for (int k = 0; k < scene->n_primitives; k++) {
        mbr_node &q = scene->node[scene->n_nodes++];
        std::memset(&q, 0, sizeof(q));
        q.type = MBR_NODE_PRIMITIVE;
        q.index = k;
        q.enabled = 1;
        q.scale = 1.0;
        q.detail_level_multiplier = 1.0;
        q.smooth_combine_distance = 0.1;
      }
      append(rep, "note: the fractal's transform makes the scene an explicit objects tree (plain engines)");
    }
  }
  for (const std::string &u : R.unsupported) append(rep, "unsupported: " + u);
  if (!R.ignored.empty()) {
    std::string s = "ignored: " + std::to_string(R.ignored.size()) + " parameters outside the DE path:";
    for (size_t i = 0; i < R.ignored.size(); i++) s += " " + R.ignored[i];
    append(rep, s);
  }
  char head[96];
  std::snprintf(head, sizeof(head), "version %.2f, %s\n", R.version, R.hybrid ? "hybrid" : "single fractal");
  rep = std::string(head) + rep;
  return finish(R.unsupported.empty() ? MBR_OK : MBR_EUNSUPPORTED);
}
