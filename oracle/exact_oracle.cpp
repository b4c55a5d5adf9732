// ORACLE — test infrastructure only.
//
// The two dense kernels of the reference's exact contraction walk, restated
// as plain loops: the outer product of two states (src/tn/exact.rs:444-480)
// and a gate applied in place (exact.rs:482-560, with the two-qubit matrix
// product of gates.rs).  Built into liboracle.so with -ffp-contract=off, so
// each complex product is re*re - im*im, re*im + im*re and each sum is
// per-component, rounded once per operation, as rustc compiles num_complex.
// oracle/exact.py walks the tree and calls these; nothing in the product
// links them.
#include <cstdint>

namespace {

struct cd {
    double re, im;
};
inline cd mul(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cd add(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }

uint64_t scatter(uint64_t index, const uint32_t* pos, uint32_t count) {
    uint64_t out = 0;
    for (uint32_t bit = 0; bit < count; ++bit)
        if ((index >> bit) & 1u) out |= uint64_t(1) << pos[bit];
    return out;
}

}  // namespace

extern "C" {

// out[scatter(li, lpos) | scatter(ri, rpos)] = left[li] * right[ri]
// (exact.rs:466-474); out has 2^(nl + nr) entries.
void oracle_exact_outer(const double* left, uint32_t nl, const uint32_t* lpos, const double* right, uint32_t nr,
                        const uint32_t* rpos, double* out) {
    const cd* l = reinterpret_cast<const cd*>(left);
    const cd* r = reinterpret_cast<const cd*>(right);
    cd* o = reinterpret_cast<cd*>(out);
    const uint64_t total = uint64_t(1) << (nl + nr);
    for (uint64_t i = 0; i < total; ++i) o[i] = {0.0, 0.0};
    for (uint64_t li = 0; li < (uint64_t(1) << nl); ++li)
        for (uint64_t ri = 0; ri < (uint64_t(1) << nr); ++ri)
            o[scatter(li, lpos, nl) | scatter(ri, rpos, nr)] = mul(l[li], r[ri]);
}

// One-qubit gate u (row-major, 4 complex) on position p of a 2^legs state
// (exact.rs:500-516).
void oracle_exact_apply_1q(double* data, uint32_t legs, uint32_t p, const double* u) {
    cd* d = reinterpret_cast<cd*>(data);
    const cd* m = reinterpret_cast<const cd*>(u);
    const uint64_t bit = uint64_t(1) << p, len = uint64_t(1) << legs;
    for (uint64_t index = 0; index < len; ++index) {
        if (index & bit) continue;
        const uint64_t up = index | bit;
        const cd v0 = d[index], v1 = d[up];
        d[index] = add(mul(m[0], v0), mul(m[1], v1));
        d[up] = add(mul(m[2], v0), mul(m[3], v1));
    }
}

// Two-qubit gate from its 4x4 matrix m[co][to][ci][ti] (16 complex) on
// control position c and target position t (exact.rs:518-544): each output
// is the four products summed left to right.
void oracle_exact_apply_2q(double* data, uint32_t legs, uint32_t c, uint32_t t, const double* m16) {
    cd* d = reinterpret_cast<cd*>(data);
    const cd* m = reinterpret_cast<const cd*>(m16);
    const uint64_t ctrl = uint64_t(1) << c, tgt = uint64_t(1) << t, len = uint64_t(1) << legs;
    auto at = [&](int co, int to, int ci, int ti) { return m[((co * 2 + to) * 2 + ci) * 2 + ti]; };
    for (uint64_t index = 0; index < len; ++index) {
        if ((index & ctrl) || (index & tgt)) continue;
        const uint64_t i_c = index | ctrl, i_t = index | tgt, i_ct = index | ctrl | tgt;
        const cd v00 = d[index], v10 = d[i_c], v01 = d[i_t], v11 = d[i_ct];
        auto amp = [&](int co, int to) {
            return add(add(add(mul(at(co, to, 0, 0), v00), mul(at(co, to, 1, 0), v10)), mul(at(co, to, 0, 1), v01)),
                       mul(at(co, to, 1, 1), v11));
        };
        const cd a00 = amp(0, 0), a10 = amp(1, 0), a01 = amp(0, 1), a11 = amp(1, 1);
        d[index] = a00;
        d[i_c] = a10;
        d[i_t] = a01;
        d[i_ct] = a11;
    }
}

// CCNOT on positions c1, c2 (controls) and t (exact.rs:546-556).
void oracle_exact_apply_ccnot(double* data, uint32_t legs, uint32_t c1, uint32_t c2, uint32_t t) {
    cd* d = reinterpret_cast<cd*>(data);
    const uint64_t m1 = uint64_t(1) << c1, m2 = uint64_t(1) << c2, mt = uint64_t(1) << t, len = uint64_t(1) << legs;
    for (uint64_t index = 0; index < len; ++index) {
        if ((index & m1) && (index & m2) && !(index & mt)) {
            const cd v = d[index];
            d[index] = d[index | mt];
            d[index | mt] = v;
        }
    }
}

}  // extern "C"
