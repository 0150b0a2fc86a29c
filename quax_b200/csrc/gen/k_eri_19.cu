// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (22|21).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(19, 2, 2, 2, 1)
