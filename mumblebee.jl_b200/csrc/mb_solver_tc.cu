// The tensor-core build of the batched solver: the same source as mb_solver.cu with the FP32
// factor's trailing-update tiles on tcgen05 (kind::tf32, 3xTF32 split, per-step FP32 read-out).
// Its kernels run one CTA per SM, as every kernel holding tcgen05 instructions does, so it is a
// separate set of kernels (names and entry points with the suffix _tc) in a namespace of its own;
// the host runtime launches it when settings.fp32_tiles asks for the tensor cores.
#define MB_TC 1
#define mb mb_tc
#include "mb_solver.cu"
