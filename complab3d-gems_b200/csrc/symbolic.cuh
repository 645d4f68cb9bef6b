// symbolic.cuh -- rate laws read from a .sym file at run time (the reference's complab3d_symbolic.hh
// language), compiled on the host into postfix code and evaluated per voxel on the device.
//
// A program is the file's rate lines in file order, each a postfix sequence over a value vector
// whose first n_vars slots are the declared variables (clamped to their ranges) and whose next
// slots are the outputs of the earlier rate lines (unscaled), exactly the scope rule of the file:
// a rate may use the variables and any earlier rate. Arithmetic is FP64 with every operation
// rounded on its own (no fused multiply-add), so a program computes what the tree of the reference
// computes, operation for operation; exp, log, log10, sqrt, tanh and pow are CUDA's.
#pragma once

#include <cstdint>

namespace clb {

constexpr int SYM_MAX_OPS = 384;     // postfix operations of all rate lines of one program
constexpr int SYM_MAX_CONST = 96;    // numeric constants
constexpr int SYM_MAX_VARS = 16;     // declared variables
constexpr int SYM_MAX_RATES = 16;    // rate lines, derived ones included
constexpr int SYM_STACK = 24;        // evaluation stack depth (checked when the program is built)
constexpr int SYM_MAX_PROGS = CLB_MAX_MICROBES + 1;  // one per microbe, then the abiotic law

enum SymOp : int16_t {
    SO_CONST, SO_VAR, SO_NEG, SO_ADD, SO_SUB, SO_MUL, SO_DIV, SO_POW, SO_EXP, SO_LOG, SO_LOG10, SO_SQRT,
    SO_ABS, SO_TANH, SO_MIN, SO_MAX
};

struct SymProg {
    int n_vars, n_rates, n_ops;
    int kind;                          // 0 biotic (a growth line), 1 abiotic (an extent line)
    double unit;                       // 1 for per_second, 1/3600 for per_hour
    int16_t op[SYM_MAX_OPS], arg[SYM_MAX_OPS];
    int16_t rate_end[SYM_MAX_RATES];   // rate r's code is [r ? rate_end[r - 1] : 0, rate_end[r])
    double cst[SYM_MAX_CONST];
    double lo[SYM_MAX_VARS], hi[SYM_MAX_VARS];  // range of each variable; hi <= lo: none
    // binding to the handle (internal species indices)
    int var_src[SYM_MAX_VARS];         // species of each variable, -1: the organism's biomass
    int rate_dst[SYM_MAX_RATES];       // species of each rate, -1: growth / extent (no species)
};

// The rates of program P for the variables x[0..n_vars): out[r] = value of rate r times the unit
// scale. A NaN rate reads as 0 and a rate beyond +-1e300 is held there (complab3d_symbolic.hh
// evaluate()). Returns true when the range clamp changed a variable.
__host__ __device__ inline bool sym_eval(const SymProg& P, const double* x, double* out) {
    double v[SYM_MAX_VARS + SYM_MAX_RATES];
    bool clamped = false;
    for (int i = 0; i < P.n_vars; ++i) {
        double a = x[i];
        if (P.hi[i] > P.lo[i]) {
            if (a < P.lo[i]) { a = P.lo[i]; clamped = true; }
            else if (a > P.hi[i]) { a = P.hi[i]; clamped = true; }
        }
        v[i] = a;
    }
    int pc = 0;
    for (int r = 0; r < P.n_rates; ++r) {
        double st[SYM_STACK];
        int sp = 0;
        for (; pc < P.rate_end[r]; ++pc) {
            const int a = P.arg[pc];
            switch (P.op[pc]) {
                case SO_CONST: st[sp++] = P.cst[a]; break;
                case SO_VAR: st[sp++] = v[a]; break;
                case SO_NEG: st[sp - 1] = -st[sp - 1]; break;
                case SO_EXP: st[sp - 1] = exp(st[sp - 1]); break;
                case SO_LOG: st[sp - 1] = st[sp - 1] > 0.0 ? log(st[sp - 1]) : 0.0; break;
                case SO_LOG10: st[sp - 1] = st[sp - 1] > 0.0 ? log10(st[sp - 1]) : 0.0; break;
                case SO_SQRT: st[sp - 1] = st[sp - 1] > 0.0 ? sqrt(st[sp - 1]) : 0.0; break;
                case SO_ABS: st[sp - 1] = fabs(st[sp - 1]); break;
                case SO_TANH: st[sp - 1] = tanh(st[sp - 1]); break;
                default: {
                    const double b = st[--sp], l = st[sp - 1];
                    double y;
                    switch (P.op[pc]) {
#ifdef __CUDA_ARCH__
                        case SO_ADD: y = __dadd_rn(l, b); break;
                        case SO_SUB: y = __dsub_rn(l, b); break;
                        case SO_MUL: y = __dmul_rn(l, b); break;
                        case SO_DIV: y = fabs(b) < 1e-300 ? 0.0 : __ddiv_rn(l, b); break;
#else
                        case SO_ADD: y = l + b; break;
                        case SO_SUB: y = l - b; break;
                        case SO_MUL: y = l * b; break;
                        case SO_DIV: y = fabs(b) < 1e-300 ? 0.0 : l / b; break;
#endif
                        case SO_POW: y = (l < 0.0 && b != floor(b)) ? 0.0 : pow(l, b); break;
                        case SO_MIN: y = l < b ? l : b; break;
                        case SO_MAX: y = l > b ? l : b; break;
                        default: y = 0.0; break;
                    }
                    st[sp - 1] = y;
                    break;
                }
            }
        }
        double y = sp > 0 ? st[sp - 1] : 0.0;
        if (y != y) y = 0.0;
        if (y > 1e300) y = 1e300;
        else if (y < -1e300) y = -1e300;
        v[P.n_vars + r] = y;
        out[r] = y * P.unit;
    }
    return clamped;
}

}  // namespace clb
