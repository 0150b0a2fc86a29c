// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.
// ERI kernels of class (21|00).
#include "../qx_kernels.cuh"
QX_DEFINE_LAUNCH(10, 2, 1, 0, 0)
