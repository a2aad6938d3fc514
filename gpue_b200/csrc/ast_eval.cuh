// ast_eval.cuh -- the postfix evaluator of GPUE expressions, host and device.
//
// Operation numbers and their meaning follow evaluate_eqn_gpu
// (src/dynamic.cu:527-603) and its helpers (src/dynamic.cu:23-160):
//   1 +  2 -  3 *  4 /  5 pow(a, (int)b)  6 cos  7 sin  8 tan  9 sqrt  10 exp
//   11 jn(a, b)  12 yn(a, b)  13 k2n(a, b)  (j0/j1 and y0/y1 for orders 0, 1)
// k2n is GPUE's poly_k series (n = 30 terms, complex pow through atan).
#pragma once

#include <cmath>

#include "ast.h"

namespace gpue {

struct AstC {
    double x, y;
};

__host__ __device__ inline AstC ast_cmul(AstC a, AstC b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

__host__ __device__ inline double ast_factorial(double v) {
    double r = v;
    if (v < 1) return 1;
    for (int i = (int)floor(v) - 1; i > 0; --i) r *= i;
    return r;
}

// complex power through modulus and atan (src/kernels.cu:12-16)
__host__ __device__ inline AstC ast_cpow(AstC a, int b) {
    const double r = sqrt(a.x * a.x + a.y * a.y);
    const double th = atan(a.y / a.x);
    return {pow(r, b) * cos(b * th), pow(r, b) * sin(b * th)};
}

__host__ __device__ inline AstC ast_poly_i(int v, AstC x, int n) {
    AstC ival = {0.0, 0.0};
    x = ast_cmul({0.0, 1.0}, x);
    for (int i = 0; i < n; ++i) {
        const double b = pow(-1.0, i) * (ast_factorial(n + i - 1) * pow((double)n, 1 - 2 * i)) /
                         (ast_factorial(i) * ast_factorial(n - i) * ast_factorial(v + i));
        AstC s = ast_cpow({x.x * 0.5, x.y * 0.5}, 2 * i + v);
        ival.x += s.x * b;
        ival.y += s.y * b;
    }
    return ival;
}

__host__ __device__ inline double ast_k2n(double a, double b) {
    const int v = (int)a, n = 30;
    AstC p = ast_poly_i(-v, {b, 0.0}, n), q = ast_poly_i(v, {b, 0.0}, n);
    const double f = 3.141592653589793 / (2 * sin(n * 3.141592653589793));
    AstC val = {(p.x - q.x) * f, (p.y - q.y) * f};
    return ast_cmul(val, val).x;
}

__host__ __device__ inline double ast_apply(int op, double a, double b) {
    switch (op) {
        case 1: return a + b;
        case 2: return a - b;
        case 3: return a * b;
        case 4: return a / b;
        case 5: return pow(a, (int)b);
        case 6: return cos(a);
        case 7: return sin(a);
        case 8: return tan(a);
        case 9: return sqrt(a);
        case 10: return exp(a);
        case 11: return ((int)a == 0) ? j0(b) : ((int)a == 1) ? j1(b) : jn((int)a, b);
        case 12: return ((int)a == 0) ? y0(b) : ((int)a == 1) ? y1(b) : yn((int)a, b);
        case 13: return ast_k2n(a, b);
        default: return 0.0;
    }
}

// Not inlined on the device: the pass kernels call it once per point from
// fully unrolled loops, and one out-of-line copy keeps their code small.
[[maybe_unused]] static __host__ __device__ __noinline__ double ast_eval(const AstInstr* prog, int n, double x,
                                                        double y, double z, double t) {
    double st[kAstMaxStack];
    int sp = 0;
    for (int i = 0; i < n; ++i) {
        const AstInstr in = prog[i];
        switch (in.code) {
            case AST_PUSH_CONST: st[sp++] = in.val; break;
            case AST_PUSH_X: st[sp++] = x; break;
            case AST_PUSH_Y: st[sp++] = y; break;
            case AST_PUSH_Z: st[sp++] = z; break;
            case AST_PUSH_T: st[sp++] = t; break;
            default: {
                const double b = st[--sp];
                const double a = st[--sp];
                st[sp++] = ast_apply(in.op_num, a, b);
            }
        }
    }
    return sp ? st[0] : 0.0;
}

}  // namespace gpue
