// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (20|11).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(8, 2, 0, 1, 1)
