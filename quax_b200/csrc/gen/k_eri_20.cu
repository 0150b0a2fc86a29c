// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (22|22).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(20, 2, 2, 2, 2)
