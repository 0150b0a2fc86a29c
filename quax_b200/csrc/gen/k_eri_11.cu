// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (21|10).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(11, 2, 1, 1, 0)
