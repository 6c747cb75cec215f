// spns_f32.cu -- the passes of one step in the compensated single-precision
// form (SPNS_FP32_HILO): transforms and products in float, the state as a
// float hi + lo pair updated in double by the spectral sweep, reductions, CFL
// and forcing normalisation in double.
#include "passes.cuh"

const PrecOps spns_ops_f32 = Passes<float>::ops();
