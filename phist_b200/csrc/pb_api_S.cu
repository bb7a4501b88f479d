// pb_api_S.cu -- phist_S* entry points (single precision, _ST_ = _MT_ = float),
// used by the mixed-precision form (FP32 sweeps and FP32 Krylov inner solves)
#include "pb_api.cuh"
#define PB_T float
#define PB_FN(name) phist_S##name
#define PB_XFN(name) phist_b200_S##name
#include "pb_api_inst.inc"
