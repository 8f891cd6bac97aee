// makea.cpp -- bit-exact NPB CG matrix generator (host C++).
//
// Produces exactly the CSR of the reference's makea()+sparse()
// (GMAP/NPB-GPU CUDA/CG/cg.cu:1303-1368, :1611-1785), seeded as main() does
// (cg.cu:404-408), but with a different construction:
//   * the LCG x <- 5^13 x mod 2^46 (CUDA/common/c_randdp.cpp:84-114) runs in
//     uint64 arithmetic: the product is taken mod 2^64, whose low 46 bits are
//     the product mod 2^46, and x * 2^-46 is exact in a double -- the same
//     numbers the reference computes with 23-bit halves in doubles;
//   * instead of the reference's ordered insertion into pre-sized row slots
//     (O(nnz * row length)), every contribution (row, col, value) is
//     bucketed by row in generation order, each row is sorted by
//     (col, generation index) and duplicates are folded left to right.  The
//     reference adds duplicate contributions in the order its loops meet them
//     (vector i, then nza, then nzrow), which is generation order, starting
//     from 0.0, so the sums are bit-identical.
//   * rows are assembled in parallel (std::thread), each thread owning a
//     contiguous row range and scanning the vectors in order.
// Built with -ffp-contract=off: products and sums must round separately, as
// in the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "cgb_internal.h"

namespace cgb {

namespace {

constexpr uint64_t kMask46 = (uint64_t(1) << 46) - 1;
constexpr uint64_t kMult = 1220703125ull;  // 5^13, main() amult (cg.cu:407)

struct Lcg46 {
    uint64_t state;
    double next()
    {
        state = (state * kMult) & kMask46;
        return std::ldexp(double(state), -46);
    }
};

using Vectors = GenVectors;  // count = arow, pos = acol (0-based), val = aelt

// n sparse vectors: nonzer distinct random positions with random values
// (sprnvc, cg.cu:1798-1833) and position i forced to 0.5 (vecset,
// cg.cu:1841-1857).
void draw_vectors(int n, int nonzer, uint64_t seed, Vectors &v)
{
    Lcg46 rng{seed};
    (void)rng.next();  // main() throws the first draw away (cg.cu:408)
    int pow2 = 1;
    do {
        pow2 *= 2;
    } while (pow2 < n);
    v.width = nonzer + 1;
    v.count.assign(n, 0);
    v.pos.assign(size_t(n) * v.width, 0);
    v.val.assign(size_t(n) * v.width, 0.0);
    std::vector<int> p1(v.width);  // 1-based positions
    std::vector<double> vv(v.width);
    for (int i = 0; i < n; i++) {
        int have = 0;
        while (have < nonzer) {
            double value = rng.next();
            double where = rng.next();
            int cand = int(pow2 * where) + 1;
            if (cand > n) continue;
            bool seen = false;
            for (int t = 0; t < have; t++)
                if (p1[t] == cand) { seen = true; break; }
            if (seen) continue;
            vv[have] = value;
            p1[have] = cand;
            have++;
        }
        bool set = false;
        for (int t = 0; t < have; t++)
            if (p1[t] == i + 1) { vv[t] = 0.5; set = true; }
        if (!set) {
            vv[have] = 0.5;
            p1[have] = i + 1;
            have++;
        }
        v.count[i] = have;
        for (int t = 0; t < have; t++) {
            v.pos[size_t(i) * v.width + t] = p1[t] - 1;
            v.val[size_t(i) * v.width + t] = vv[t];
        }
    }
}

// Assemble rows [r0, r1): bucket the contributions of every vector that
// touches these rows, in generation order, then sort and fold each row.
// Writes unique entries per row into (ucol, uval) at ubase[row] and the
// count into ucount[row].
struct RowJob {
    int r0, r1;
};

void assemble_rows(const Vectors &v, const std::vector<double> &scale_of, int n, double rcond,
                   double shift, const std::vector<long long> &slot, RowJob job,
                   std::vector<int> &bcol, std::vector<double> &bval, std::vector<int> &ucount)
{
    const int w = v.width;
    // fill cursor per row, relative to slot[row]
    std::vector<long long> cursor(size_t(job.r1 - job.r0), 0);
    for (int i = 0; i < n; i++) {
        const int cnt = v.count[i];
        const int *pos = &v.pos[size_t(i) * w];
        const double *val = &v.val[size_t(i) * w];
        for (int s = 0; s < cnt; s++) {
            const int row = pos[s];
            if (row < job.r0 || row >= job.r1) continue;
            const double scale = scale_of[i] * val[s];
            long long at = slot[row] + cursor[row - job.r0];
            for (int u = 0; u < cnt; u++) {
                const int col = pos[u];
                double va = val[u] * scale;
                if (col == row && row == i) {
                    va = va + rcond;
                    va = va - shift;
                }
                bcol[at] = col;
                bval[at] = va;
                at++;
            }
            cursor[row - job.r0] += cnt;
        }
    }
    // sort each row by (col, generation index) and fold duplicates in order
    std::vector<uint64_t> key;
    std::vector<int> tcol;
    std::vector<double> tval;
    for (int row = job.r0; row < job.r1; row++) {
        const long long b = slot[row], e = slot[row + 1];
        const int len = int(e - b);
        key.resize(len);
        for (int t = 0; t < len; t++) key[t] = (uint64_t(uint32_t(bcol[b + t])) << 32) | uint32_t(t);
        std::sort(key.begin(), key.end());
        tcol.resize(len);
        tval.resize(len);
        int u = -1;
        for (int t = 0; t < len; t++) {
            const int col = int(key[t] >> 32);
            const double va = bval[b + int(key[t] & 0xffffffffu)];
            if (u >= 0 && tcol[u] == col) {
                tval[u] = tval[u] + va;
            } else {
                u++;
                tcol[u] = col;
                tval[u] = 0.0;
                tval[u] = tval[u] + va;
            }
        }
        const int uniq = u + 1;
        for (int t = 0; t < uniq; t++) {
            bcol[b + t] = tcol[t];
            bval[b + t] = tval[t];
        }
        ucount[row] = uniq;
    }
}

unsigned worker_count(int n)
{
    unsigned hw = std::thread::hardware_concurrency();
    if (hw == 0) hw = 1;
    unsigned want = unsigned(std::max(1, n / 2000));
    return std::max(1u, std::min(hw, std::min(want, 64u)));
}

}  // namespace

int draw_generator_vectors(int n, int nonzer, double rcond, double seed, GenVectors &v)
{
    if (n < 2 || nonzer < 1 || nonzer >= n)
        return set_error(CGB_ERR_INVALID, "makea: need n >= 2, 1 <= nonzer < n");
    if (!valid_seed(seed))
        return set_error(CGB_ERR_INVALID, "makea: seed must be an odd integer in (1, 2^46)");
    try {
        draw_vectors(n, nonzer, uint64_t(seed), v);
        // geometric scale per vector: size *= ratio after each (cg.cu:1695, :1755)
        v.scale.resize(n);
        const double ratio = std::pow(rcond, 1.0 / double(n));
        double size = 1.0;
        for (int i = 0; i < n; i++) {
            v.scale[i] = size;
            size = size * ratio;
        }
    } catch (const std::bad_alloc &) {
        return set_error(CGB_ERR_NOMEM, "makea: host allocation failed");
    }
    return CGB_OK;
}

bool valid_seed(double seed)
{
    if (!(seed > 1.0) || !(seed < 70368744177664.0)) return false;  // (1, 2^46)
    if (std::floor(seed) != seed) return false;
    return (uint64_t(seed) & 1u) == 1u;
}

int makea(int n, int nonzer, double rcond, double shift, double seed, int *rowstr, int *colidx,
          double *a, long long cap, long long *nnz_out)
{
    if (n < 2 || nonzer < 1 || nonzer >= n || !rowstr || !nnz_out)
        return set_error(CGB_ERR_INVALID, "makea: need n >= 2, 1 <= nonzer < n, non-null outputs");
    if (!valid_seed(seed))
        return set_error(CGB_ERR_INVALID, "makea: seed must be an odd integer in (1, 2^46)");
    if (!(rcond > 0.0) || !std::isfinite(shift))
        return set_error(CGB_ERR_INVALID, "makea: rcond must be > 0 and shift finite");
    try {
        Vectors v;
        const int vst = draw_generator_vectors(n, nonzer, rcond, seed, v);
        if (vst) return vst;
        const std::vector<double> &scale_of = v.scale;

        // contributions per row (cg.cu:1649-1662) and their offsets
        std::vector<long long> slot(size_t(n) + 1, 0);
        for (int i = 0; i < n; i++)
            for (int s = 0; s < v.count[i]; s++) slot[v.pos[size_t(i) * v.width + s] + 1] += v.count[i];
        for (int j = 0; j < n; j++) slot[j + 1] += slot[j];
        const long long total = slot[n];

        std::vector<int> bcol(static_cast<size_t>(total));
        std::vector<double> bval(static_cast<size_t>(total));
        std::vector<int> ucount(static_cast<size_t>(n), 0);

        const unsigned nw = worker_count(n);
        // split rows so each worker gets about the same number of contributions
        std::vector<RowJob> jobs;
        int r = 0;
        for (unsigned wk = 0; wk < nw; wk++) {
            long long target = (total * (long long)(wk + 1)) / (long long)nw;
            int r1 = r;
            while (r1 < n && slot[r1] < target) r1++;
            if (wk + 1 == nw) r1 = n;
            jobs.push_back({r, r1});
            r = r1;
        }
        std::vector<std::thread> pool;
        for (size_t t = 1; t < jobs.size(); t++)
            pool.emplace_back(assemble_rows, std::cref(v), std::cref(scale_of), n, rcond, shift,
                              std::cref(slot), jobs[t], std::ref(bcol), std::ref(bval),
                              std::ref(ucount));
        assemble_rows(v, scale_of, n, rcond, shift, slot, jobs[0], bcol, bval, ucount);
        for (auto &th : pool) th.join();

        long long nnz = 0;
        for (int j = 0; j < n; j++) nnz += ucount[j];
        *nnz_out = nnz;
        if (nnz > cap)
            return set_error(CGB_ERR_CAPACITY, "makea: nz_capacity %lld < nnz %lld", cap, nnz);
        if (nnz > 0x7fffffffLL)
            return set_error(CGB_ERR_CAPACITY, "makea: nnz %lld overflows int32 rowstr", nnz);
        if (!colidx || !a) return set_error(CGB_ERR_INVALID, "makea: null colidx/a");
        long long out = 0;
        rowstr[0] = 0;
        for (int j = 0; j < n; j++) {
            std::memcpy(colidx + out, &bcol[slot[j]], sizeof(int) * size_t(ucount[j]));
            std::memcpy(a + out, &bval[slot[j]], sizeof(double) * size_t(ucount[j]));
            out += ucount[j];
            rowstr[j + 1] = int(out);
        }
        return CGB_OK;
    } catch (const std::bad_alloc &) {
        return set_error(CGB_ERR_NOMEM, "makea: host allocation failed");
    }
}

}  // namespace cgb
