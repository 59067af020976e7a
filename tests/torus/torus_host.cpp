// Host build of the library's Fishbone-Moncrief torus context (rt_torus.cuh),
// for the CPU check against the oracle's restatement.  Test-only.
#include "rt_torus.cuh"

extern "C" void host_torus(double mass, double spin, double r_in_units, double r_center_units, double out[9]) {
    const relsim::torus::TorusContext c = relsim::torus::make_torus(mass, spin, r_in_units, r_center_units);
    out[0] = c.valid ? 1.0 : 0.0;
    out[1] = c.closed ? 1.0 : 0.0;
    out[2] = c.h_max;
    out[3] = c.inner_bound;
    out[4] = c.outer_bound;
    out[5] = c.t.l;
    out[6] = c.t.w_in;
    out[7] = c.t.a;
    out[8] = c.t.rh;
}

// Enthalpy and fluid four-velocity at (r, theta) of that torus.
extern "C" void host_torus_fluid(double mass, double spin, double r_in_units, double r_center_units, double r,
                                 double theta, double out[3]) {
    const relsim::torus::TorusContext c = relsim::torus::make_torus(mass, spin, r_in_units, r_center_units);
    out[0] = relsim::torus::enthalpy(c.t, r, theta);
    relsim::torus::four_velocity(c.t, r, theta, out[1], out[2]);
}
