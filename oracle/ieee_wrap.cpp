/*
 * C entry points of the reference's IEEE field evaluator.  TEST INFRASTRUCTURE
 * ONLY.  oracle/Makefile compiles the reference's
 * sandbox/ieee_hyperbolic/ieee_hyperbolic.cpp unmodified, in place (its main()
 * renamed on the command line so the file links into a shared library), with
 * this file into _ref/libd4ref_ieee.so.  IEEE_xy / IEEE_xy_diff_x
 * (ieee_hyperbolic.cpp:103-140) are the exact truncated image sums of
 * src/Fields/Field.cpp:26-168 (USE_IEEE_HYPERBOLIC 1).
 */
double IEEE_xy(double dx, double dy);
double IEEE_xy_diff_x(double dx, double dy);

extern "C" double d4ref_ieee_xy(double dx, double dy) { return IEEE_xy(dx, dy); }
extern "C" double d4ref_ieee_xy_diff_x(double dx, double dy) { return IEEE_xy_diff_x(dx, dy); }
