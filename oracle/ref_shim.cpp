/*
 * ref_shim.cpp -- C entry points around the reference's own CPU functions.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles this file in one
 * translation unit after the CPU loops it takes, at build time, straight
 * from the reference sources (src/main8.cu:49-103 into namespace ref8,
 * src/main9.cu:48-69 into namespace ref9); the result goes only to
 * oracle/_ref/libmgvref.so, which tests use to pin the oracle and to make
 * the golden fixtures.  No reference source text is stored in this repo.
 *
 * The reference keeps its state in globals (hist[5001], ht[1 << 20]) and
 * never resets them between calls (src/main8.cu:55,72-73); each wrapper
 * resets them first so that every call stands alone.
 */
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {

/* stable_select_cpu with a threshold (src/main9.cu:48-52): count of rows
 * with a[i] <= thres; the selected values are written to out if non-NULL. */
unsigned long long mgvref_stable_select(const int32_t *a, int32_t *out, size_t n, int32_t thres) {
    std::vector<int32_t> tmp(n ? n : 1);
    size_t k = ref9::stable_select_cpu(const_cast<int32_t *>(a), tmp.data(), n, thres);
    if (out) std::memcpy(out, tmp.data(), k * sizeof(int32_t));
    return (unsigned long long)k;
}

/* sum_select_cpu with a threshold (src/main9.cu:56-61): wrapping int32
 * SUM of the selected values. */
int32_t mgvref_sum_select(const int32_t *a, size_t n, int32_t thres) {
    int32_t b[1] = {0};
    ref9::sum_select_cpu(const_cast<int32_t *>(a), b, n, thres);
    return b[0];
}

/* sum_selfjoin_select_cpu (src/main8.cu:64-70): wrapping int32 of
 * sum over v in 1..5000 of hist[v]^2 for rows a <= 5000. */
int32_t mgvref_sum_selfjoin_select(const int32_t *a, int n) {
    std::memset(ref8::hist, 0, sizeof(ref8::hist));
    int32_t b[1] = {0};
    ref8::sum_selfjoin_select_cpu(const_cast<int32_t *>(a), b, n);
    return b[0];
}

/* sum_hashjoin_select_cpu (src/main8.cu:84-103): builds a chained table
 * over the rows of a with a <= 5000 (2^20 buckets, murmur finaliser) and
 * counts, as a wrapping int32, the probe rows' matches. */
int32_t mgvref_sum_hashjoin_select(const int32_t *a, int n, const int32_t *probe, int m) {
    for (int i = 0; i < (1 << ref8::log_htsize); ++i) ref8::ht[i] = -1;
    std::vector<int32_t> next(n ? n : 1);
    int32_t b[1] = {0};
    ref8::sum_hashjoin_select_cpu(const_cast<int32_t *>(a), b, const_cast<int32_t *>(probe),
                                  next.data(), n, m);
    return b[0];
}

/* h_hashMurmur (src/main8.cu:75-82): finaliser masked to 2^20 buckets. */
uint32_t mgvref_hash_murmur_masked(uint32_t x) { return ref8::h_hashMurmur(x); }

int mgvref_log_htsize(void) { return ref8::log_htsize; }

}  /* extern "C" */
