// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (11|00).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(3, 1, 1, 0, 0)
