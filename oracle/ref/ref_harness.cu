// ref_harness.cu — TEST INFRASTRUCTURE: runs the reference's own
// AriesDecimal<LEN> arithmetic (src/datatypes/AriesDecimal.hxx) on the GPU so
// the tests can pin the CPU oracle and the CUDA path to the reference.
//
// Built by oracle/ref/Makefile from the reference sources where they lie;
// only this driver (kernels that mirror the reference's generated kernel text,
// AriesExprCalcNode.cpp:1285-1428) is written here.
//
// Safety (nothing here may fault or hang a GPU):
//   * the reference's multiply writes one limb past its result array
//     (AriesDecimal.hxx:397-401) and its decimal shift reads/writes one past
//     (:128-136); every evaluation runs in a non-inlined function called from
//     a kernel frame that keeps a stack pad above it, so such writes land in
//     the pad;
//   * its chunked long division loops until a shift count reaches zero and
//     only makes progress when the dividend leaves two spare limbs
//     (:796-823); the host entry refuses limb counts without that headroom;
//   * its power-of-ten table stops at 10^38 (:12-63); the host entry refuses
//     alignment or divide shifts above 38.
#include <cuda_runtime.h>
#include <stdint.h>

#include "AriesDefinition.h"
#include "datatypes/decimal.hxx"
#include "datatypes/AriesDecimal.hxx"

BEGIN_ARIES_ACC_NAMESPACE

// the table text is extracted from decimal.cu:92 by the build recipe
#define REF_PREC_BYTES_INIT
static const uint32_t h_ref_prec_bytes[] =
#include "ref_prec_bytes.inc"
;
__device__ static const uint32_t d_ref_prec_bytes[] =
#include "ref_prec_bytes.inc"
;

// GetDecimalRealBytes (decimal.cu:464-467) over the same table.
ARIES_HOST_DEVICE_NO_INLINE int GetDecimalRealBytes(uint16_t precision, uint16_t scale) {
#ifdef __CUDA_ARCH__
    return (int)d_ref_prec_bytes[precision];
#else
    return (int)h_ref_prec_bytes[precision];
#endif
}

END_ARIES_ACC_NAMESPACE

using aries_acc::AriesDecimal;
using aries_acc::CompactDecimal;

enum { OP_ADD = 0, OP_SUB = 1, OP_MUL = 2, OP_DIV = 3, OP_MOD = 4, OP_MAD = 20, OP_Q_DP = 30, OP_Q_CHARGE = 31 };

struct Args {
    int op;
    const char* a;
    const char* b;
    const char* c;
    int pa, sa, pb, sb, pc, sc;
    int ba, bb, bc;
    int64_t rows;
    char* out;
    int ob;
};

template <int LEN>
__device__ __noinline__ void eval_row(const Args& g, int64_t i) {
    AriesDecimal<LEN> x((CompactDecimal*)(g.a + i * g.ba), g.pa, g.sa);
    AriesDecimal<LEN> y((CompactDecimal*)(g.b + i * g.bb), g.pb, g.sb);
    char* o = g.out + i * g.ob;
    if (g.op >= 10 && g.op <= 15) {
        bool r;
        switch (g.op) {
            case 10: r = x < y; break;
            case 11: r = x <= y; break;
            case 12: r = x > y; break;
            case 13: r = x >= y; break;
            case 14: r = x == y; break;
            default: r = !(x == y); break;
        }
        o[0] = r ? 1 : 0;
        return;
    }
    AriesDecimal<LEN> r;
    switch (g.op) {
        case OP_ADD: r = x + y; break;
        case OP_SUB: r = x - y; break;
        case OP_MUL: r = x * y; break;
        case OP_DIV: r = x / y; break;
        case OP_MOD: r = x % y; break;
        case OP_MAD: {
            // the generated text after AlignOptimize: (c + (a * b))
            AriesDecimal<LEN> z((CompactDecimal*)(g.c + i * g.bc), g.pc, g.sc);
            r = z + (x * y);
            break;
        }
        case OP_Q_DP:
        case OP_Q_CHARGE: {
            // price * (1.00 - disc) [* (1.00 + tax)]: x = price, y = disc, z = tax
            AriesDecimal<LEN> one;
            one.v[0] = 100;
            one.frac = 2;
            r = x * (one - y);
            if (g.op == OP_Q_CHARGE) {
                AriesDecimal<LEN> z((CompactDecimal*)(g.c + i * g.bc), g.pc, g.sc);
                r = r * (one + z);
            }
            break;
        }
        default: break;
    }
    r.ToCompactDecimal(o, g.ob);
}

template <int LEN>
__global__ void k_eval(Args g) {
    volatile uint32_t pad[64];  // stack headroom above eval_row's frame
    pad[threadIdx.x & 63] = threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.rows; i += stride) eval_row<LEN>(g, i);
    if (pad[threadIdx.x & 63] == 0xffffffffu) g.out[0] = 0;
}

template <int LEN>
static int launch(const Args& g) {
    int64_t blocks = (g.rows + 127) / 128;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    k_eval<LEN><<<(unsigned)blocks, 128>>>(g);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

extern "C" int ref_max_shift() { return 38; }

// Limb counts instantiated (each compiles the reference's full operator set).
extern "C" int ref_supported_len(int len) {
    switch (len) {
        case 2: case 3: case 4: case 5: case 6: case 8: case 10: case 12: case 16: case 20: case 24: case 32:
            return 1;
        default:
            return 0;
    }
}

// Evaluate one operator (or the fixed shapes above) with AriesDecimal<len>.
// All pointers are device pointers.  Returns 0, -1 for an unsupported len,
// -2 for a request outside the reference's safe domain, else a CUDA error.
extern "C" int ref_eval(int op, int len, const void* a, int pa, int sa, const void* b, int pb, int sb, const void* c,
                        int pc, int sc, int64_t rows, void* out, int out_bytes, int need_limbs) {
    if (!ref_supported_len(len)) return -1;
    if (need_limbs + 2 > len) return -2;  // two spare limbs: the long-division loop needs them
    if (out_bytes > 4 * len) return -2;   // ToCompactDecimal copies out_bytes from the limb array
    const int sd = sa > sb ? sa - sb : sb - sa;
    if (sd > 38) return -2;
    if ((op == OP_DIV) && sb + 4 > 38) return -2;
    if (op == OP_MAD && (sc > sa + sb ? sc - sa - sb : sa + sb - sc) > 38) return -2;
    Args g;
    g.op = op;
    g.a = (const char*)a;
    g.b = (const char*)b;
    g.c = (const char*)c;
    g.pa = pa; g.sa = sa; g.pb = pb; g.sb = sb; g.pc = pc; g.sc = sc;
    g.ba = aries_acc::h_ref_prec_bytes[pa];
    g.bb = aries_acc::h_ref_prec_bytes[pb];
    g.bc = c ? aries_acc::h_ref_prec_bytes[pc] : 0;
    g.rows = rows;
    g.out = (char*)out;
    g.ob = out_bytes;
    if (rows <= 0) return 0;
    switch (len) {
        case 2: return launch<2>(g);
        case 3: return launch<3>(g);
        case 4: return launch<4>(g);
        case 5: return launch<5>(g);
        case 6: return launch<6>(g);
        case 8: return launch<8>(g);
        case 10: return launch<10>(g);
        case 12: return launch<12>(g);
        case 16: return launch<16>(g);
        case 20: return launch<20>(g);
        case 24: return launch<24>(g);
        case 32: return launch<32>(g);
        default: return -1;
    }
}
