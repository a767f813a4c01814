/*
 * index_wrap.h -- lets the reference's periodic index wrap build for NX, NY that are
 * not powers of two (384, 96, 192), without editing its sources.  TEST INFRASTRUCTURE
 * ONLY (oracle/_ref/).
 *
 * The wrap functions (staggered/data_global_inc.h:4-7, collocated_AB3/data_global.h:1-4)
 * test `j & (NX-1)` and `j & (NX*(NY-1))`.  For powers of two these are j % NX and
 * NX*((j/NX) % NY): the x index of cell j, and the y index times NX.  Here NX and NY are
 * prvalues of small literal types that convert to int wherever the reference uses them
 * as numbers (sizes, loops, FFT plans, launch grids); only the two mask expressions,
 * NX - 1 and NX * (NY - 1) on the right of `&`, resolve to the overloaded operators
 * below, which return those modular forms.  For powers of two the result is the same
 * as the bitmask's, so the reference's arithmetic is otherwise untouched.  This is the
 * "minimal non-power-of-two index-wrap patch", made at compile time.
 */
#ifndef TCREF_INDEX_WRAP_H
#define TCREF_INDEX_WRAP_H

#if defined(__CUDACC__)
#define TCREF_HD __host__ __device__
#else
#define TCREF_HD
#endif

struct tcref_nx_t {
    TCREF_HD constexpr operator int() const { return REF_NX; }
};
struct tcref_ny_t {
    TCREF_HD constexpr operator int() const { return REF_NY; }
};
struct tcref_nx_less_t {  // NX - k
    int v;
    TCREF_HD constexpr operator int() const { return v; }
};
struct tcref_ny_less_t {  // NY - k
    int v;
    TCREF_HD constexpr operator int() const { return v; }
};
struct tcref_ymask_t {  // NX * (NY - k)
    int v, ny_less;
    TCREF_HD constexpr operator int() const { return v; }
};

TCREF_HD constexpr tcref_nx_less_t operator-(tcref_nx_t, int k) { return tcref_nx_less_t{REF_NX - k}; }
TCREF_HD constexpr tcref_ny_less_t operator-(tcref_ny_t, int k) { return tcref_ny_less_t{REF_NY - k}; }
TCREF_HD constexpr tcref_ymask_t operator*(tcref_nx_t, tcref_ny_less_t m) {
    return tcref_ymask_t{REF_NX * m.v, m.v};
}
// j & (NX - 1): the x index of cell j (j >= 0 at every call site)
TCREF_HD constexpr int operator&(int j, tcref_nx_less_t m) { return m.v == REF_NX - 1 ? j % REF_NX : (j & m.v); }
// j & (NX * (NY - 1)): NX times the y index of cell j
TCREF_HD constexpr int operator&(int j, tcref_ymask_t m) {
    return m.ny_less == REF_NY - 1 ? REF_NX * ((j / REF_NX) % REF_NY) : (j & m.v);
}

#define NX (tcref_nx_t{})
#define NY (tcref_ny_t{})

#endif
