// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (22|20).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(18, 2, 2, 2, 0)
