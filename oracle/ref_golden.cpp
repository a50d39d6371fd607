// ref_golden.cpp — golden vectors from the reference's own host-compilable code.
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile (target `ref`) into
// oracle/_ref/ref_golden, with the reference's include tree on the include path
// (the reference is not copied). It evaluates the reference's complex
// arithmetic (compas/core/complex_type.h: exp :106-114, polar :89-99,
// pow :153-161, fma :174-178, operator* :220-223) in FP32 on seeded inputs and
// prints JSON; tests/golden/make_golden.py stores the output as
// tests/golden/ref_complex_ops.json. These are the primitives the oracle's FP32
// twin builds the signal / Jacobian / EPG formulas from.
#include <cstdio>
#include <random>

#include "compas/core/complex_type.h"

using compas::cfloat;

int main() {
    std::mt19937_64 rng(20241203);
    std::uniform_real_distribution<float> ure(-3.0f, 1.0f), uim(-60.0f, 60.0f), u1(-2.0f, 2.0f),
        upow(0.0f, 250.0f);
    const int n = 64;
    std::printf("{\n");
    // exp(z)
    std::printf("\"exp\": [");
    for (int i = 0; i < n; i++) {
        cfloat z(ure(rng), uim(rng));
        cfloat e = compas::exp(z);
        std::printf("%s[%.9g, %.9g, %.9g, %.9g]", i ? ", " : "", z.re, z.im, e.re, e.im);
    }
    std::printf("],\n");
    // pow(a, b) with |a| < 1 (per-sample decay step) and integer-valued b (sample index)
    std::printf("\"pow\": [");
    for (int i = 0; i < n; i++) {
        cfloat a = compas::exp(cfloat(-std::abs(u1(rng)) * 0.01f, u1(rng)));
        float b = float(int(upow(rng)));
        cfloat p = compas::pow(a, b);
        std::printf("%s[%.9g, %.9g, %.9g, %.9g, %.9g]", i ? ", " : "", a.re, a.im, b, p.re, p.im);
    }
    std::printf("],\n");
    // fma(a, b, c) = c + a*b
    std::printf("\"fma\": [");
    for (int i = 0; i < n; i++) {
        cfloat a(u1(rng), u1(rng)), b(u1(rng), u1(rng)), c(u1(rng), u1(rng));
        cfloat r = compas::fma(a, b, c);
        std::printf("%s[%.9g, %.9g, %.9g, %.9g, %.9g, %.9g, %.9g, %.9g]", i ? ", " : "", a.re, a.im, b.re, b.im,
                    c.re, c.im, r.re, r.im);
    }
    std::printf("],\n");
    // a * b
    std::printf("\"mul\": [");
    for (int i = 0; i < n; i++) {
        cfloat a(u1(rng), u1(rng)), b(u1(rng), u1(rng));
        cfloat r = a * b;
        std::printf("%s[%.9g, %.9g, %.9g, %.9g, %.9g, %.9g]", i ? ", " : "", a.re, a.im, b.re, b.im, r.re, r.im);
    }
    std::printf("]\n}\n");
    return 0;
}
