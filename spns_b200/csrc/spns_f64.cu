// spns_f64.cu -- the passes of one step in double precision (SPNS_FP64).
#include "passes.cuh"

const PrecOps spns_ops_f64 = Passes<double>::ops();
