// Layout conversion between a plan's packed field and the reference CUDA solver's on-disk layout.
//
// The CUDA solver's files (.ics initial conditions, .plas frame series) hold the 9 components of
// beta^P in the order xx xy xz yx yy yz zx zy zz, each component with grid axis 0 fastest: the
// reference writes every component transposed (Plasticity/RunCUDA.py L9-22, convertStateToCUDA)
// and LoadStateRaw transposes back on read (Plasticity/FieldInitializers/FieldInitializer.py
// L61-103). A plan stores each component with the last axis contiguous. So element
// (i0, i1, i2) of a component sits at i0 + n0 (i1 + n1 i2) in a file and at (i0 n1 + i1) n2 + i2
// in a plan; a 2-D grid (n0, n1) is the 3-D case (n0, 1, n1). Each block moves one 32 x 32 tile
// of the (i0, i2) plane at fixed (component, i1) through shared memory, reading and writing whole
// 128-byte rows on both sides, and converts the precision on the way (FP64 <-> FP32 rounds to
// nearest, as numpy's astype).
#include "cdd_internal.cuh"

namespace cdd {

constexpr int XT = 32;          // tile edge
constexpr int XROWS = 8;        // thread rows per block (blockDim = 32 x 8)

// TO_FILE false: src in the file layout, dst in the plan layout; true: the reverse.
template <bool TO_FILE, typename S, typename D>
__global__ void __launch_bounds__(XT * XROWS) k_field_xpose(const S* __restrict__ src, D* __restrict__ dst,
                                                            int n0, int n1, int n2) {
    __shared__ D tile[XT][XT + 1];
    const int tiles0 = (n0 + XT - 1) / XT;
    const int t0 = blockIdx.x % tiles0, t2 = blockIdx.x / tiles0;
    const int i1 = blockIdx.y, c = blockIdx.z;
    const long long cells = (long long)n0 * n1 * n2;
    const S* s = src + c * cells;
    D* d = dst + c * cells;
    const int tx = threadIdx.x;
    if (!TO_FILE) {
        // read rows of the file layout (i0 fastest), write rows of the plan layout (i2 fastest)
        for (int r = threadIdx.y; r < XT; r += XROWS) {
            const int i0 = t0 * XT + tx, i2 = t2 * XT + r;
            if (i0 < n0 && i2 < n2) tile[r][tx] = (D)s[i0 + (long long)n0 * (i1 + (long long)n1 * i2)];
        }
        __syncthreads();
        for (int r = threadIdx.y; r < XT; r += XROWS) {
            const int i2 = t2 * XT + tx, i0 = t0 * XT + r;
            if (i0 < n0 && i2 < n2) d[((long long)i0 * n1 + i1) * n2 + i2] = tile[tx][r];
        }
    } else {
        for (int r = threadIdx.y; r < XT; r += XROWS) {
            const int i2 = t2 * XT + tx, i0 = t0 * XT + r;
            if (i0 < n0 && i2 < n2) tile[r][tx] = (D)s[((long long)i0 * n1 + i1) * n2 + i2];
        }
        __syncthreads();
        for (int r = threadIdx.y; r < XT; r += XROWS) {
            const int i0 = t0 * XT + tx, i2 = t2 * XT + r;
            if (i0 < n0 && i2 < n2) d[i0 + (long long)n0 * (i1 + (long long)n1 * i2)] = tile[tx][r];
        }
    }
}

template <bool TO_FILE, typename S, typename D>
static cudaError_t xpose(const void* src, void* dst, int n0, int n1, int n2, cudaStream_t st) {
    const long long tiles = (long long)((n0 + XT - 1) / XT) * ((n2 + XT - 1) / XT);
    if (tiles > 0x7fffffffLL || n1 > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)tiles, (unsigned)n1, 9);
    k_field_xpose<TO_FILE, S, D><<<grid, dim3(XT, XROWS), 0, st>>>((const S*)src, (D*)dst, n0, n1, n2);
    return cudaGetLastError();
}

cudaError_t launch_field_xpose(bool to_file, const void* src, int src_prec, void* dst, int dst_prec, int n0, int n1,
                               int n2, cudaStream_t st) {
    const bool s64 = (src_prec == CDD_F64), d64 = (dst_prec == CDD_F64);
    if (to_file) {
        if (s64 && d64) return xpose<true, double, double>(src, dst, n0, n1, n2, st);
        if (s64) return xpose<true, double, float>(src, dst, n0, n1, n2, st);
        if (d64) return xpose<true, float, double>(src, dst, n0, n1, n2, st);
        return xpose<true, float, float>(src, dst, n0, n1, n2, st);
    }
    if (s64 && d64) return xpose<false, double, double>(src, dst, n0, n1, n2, st);
    if (s64) return xpose<false, double, float>(src, dst, n0, n1, n2, st);
    if (d64) return xpose<false, float, double>(src, dst, n0, n1, n2, st);
    return xpose<false, float, float>(src, dst, n0, n1, n2, st);
}

}  // namespace cdd
