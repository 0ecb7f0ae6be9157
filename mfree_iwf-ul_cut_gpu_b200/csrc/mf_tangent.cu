// Differentiable form: the FP64 leap-frog step (leap_frog.cu:94-155) carried out on dual
// numbers, so that every state variable also carries its derivatives with respect to one, or
// all six, of the Johnson-Cook parameters A, B, n, C, m and the friction coefficient mu. Forward-mode
// (tangent) propagation: the derivative of the window-averaged tool force follows the state
// through every step, the cell-list sort included (a permutation), with no checkpoints.
//
// The kernels restate the step of mf_kernels.cuh in dual arithmetic, one thread per particle,
// in the reference's order of operations: gather + predictor + EOS + artificial stress, the
// pair sums over the 5x5 window with the rates, and the corrector .. boundary conditions with
// the secant return map iterated on duals. The cell lists come from the product's own
// kernels (k_hash_count, k_scan, k_scatter and the stable rank) run on the value positions.
// Supported: locked grid (Green order), Brookshaw or no heat conduction, the Johnson-Cook law.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "mf_dual.cuh"
#include "mf_kernels.cuh"
#include "mfree_b200.h"

// one direction (the parameter chosen per call) in mf::tg, all six at once in mf::tg6
#define MF_TG_ND 1
#define MF_TG_NS tg
#include "mf_tangent_impl.cuh"
#undef MF_TG_NS
#undef MF_TG_ND
#define MF_TG_ND 6
#define MF_TG_NS tg6
#include "mf_tangent_impl.cuh"
#undef MF_TG_NS
#undef MF_TG_ND
