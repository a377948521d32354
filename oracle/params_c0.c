/*
 * Compile-time parameter set for the 2D droplet workload (128 x 128, uniform
 * x, no buoyancy, zero wall temperature).  TEST INFRASTRUCTURE ONLY: it
 * replaces the reference's src/param/{buoyancy,boundary-condition,implicit}.c
 * when the reference is compiled into the oracle library "libsvof_ref_c0".
 * The reference fixes these values at compile time (include/param.h:10-34);
 * buoyancy on and wall temperatures +-0.5 are its defaults
 * (src/param/buoyancy.c:3, src/param/boundary-condition.c:3-6).
 */
#include "param.h"

const bool param_add_buoyancy = false;

const bool param_m_implicit_x = true;
const bool param_m_implicit_y = false;
const bool param_t_implicit_x = true;
const bool param_t_implicit_y = false;

const double param_uy_xm = 0.;
const double param_uy_xp = 0.;
const double param_t_xm = 0.;
const double param_t_xp = 0.;
