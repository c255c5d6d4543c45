/*
 * TEST ORACLE ONLY — plain-C restatement of the reference's CPU algorithm for the SPH-VE hydro step (see
 * sph_oracle.h). FP64 throughout, compiled with -ffp-contract=off so every expression rounds as written.
 * Citations are files of the reference project (tischwab0911/sphexa).
 */
#define _GNU_SOURCE
#include "sph_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX_LEVEL 21
#define ROOT_RANGE (UINT64_C(1) << 63)
#define REMOVE_KEY (UINT64_C(1) << 63)

/* ---------------------------------------------------------------------------------------------------------------- */
/* SFC keys: cstone/sfc/hilbert.hpp:43-94 (iHilbert), cstone/sfc/sfc.hpp:141-178 (sfc3D), :267-275 (batch)          */
/* ---------------------------------------------------------------------------------------------------------------- */

uint64_t orc_hilbert(unsigned px, unsigned py, unsigned pz)
{
    static const unsigned toHilbert[8] = {0, 1, 3, 2, 7, 6, 4, 5};
    uint64_t key = 0;
    for (int level = MAX_LEVEL - 1; level >= 0; --level)
    {
        unsigned xi = (px >> level) & 1u, yi = (py >> level) & 1u, zi = (pz >> level) & 1u;
        key         = (key << 3) + toHilbert[(xi << 2) | (yi << 1) | zi];
        px ^= 0u - (xi & ((!yi) | zi));
        py ^= 0u - ((xi & (yi | zi)) | (yi & (!zi)));
        pz ^= 0u - ((xi & (!yi) & (!zi)) | (yi & (!zi)));
        if (zi)
        {
            unsigned t = px;
            px         = py;
            py         = pz;
            pz         = t;
        }
        else if (!yi)
        {
            unsigned t = px;
            px         = pz;
            pz         = t;
        }
    }
    return key;
}

/* inverse of orc_hilbert: from the finest digit up, undo each level's permutation and reflection on the lower bits */
void orc_hilbert_decode(uint64_t key, unsigned* ix, unsigned* iy, unsigned* iz)
{
    static const unsigned toMorton[8] = {0, 1, 3, 2, 6, 7, 5, 4};
    unsigned px = 0, py = 0, pz = 0;
    for (unsigned level = 0; level < MAX_LEVEL; ++level)
    {
        unsigned oct = toMorton[(key >> (3 * level)) & 7u];
        unsigned xi = oct >> 2, yi = (oct >> 1) & 1u, zi = oct & 1u;
        unsigned mask = (1u << level) - 1u;
        if (zi)
        {
            unsigned t = pz;
            pz         = py;
            py         = px;
            px         = t;
        }
        else if (!yi)
        {
            unsigned t = px;
            px         = pz;
            pz         = t;
        }
        px ^= mask & (0u - (xi & ((!yi) | zi)));
        py ^= mask & (0u - ((xi & (yi | zi)) | (yi & (!zi))));
        pz ^= mask & (0u - ((xi & (!yi) & (!zi)) | (yi & (!zi))));
        px |= xi << level;
        py |= yi << level;
        pz |= zi << level;
    }
    *ix = px;
    *iy = py;
    *iz = pz;
}

static unsigned quantise(double x, double lo, double hi)
{
    const int mcoord = (1 << MAX_LEVEL) - 1;
    double m         = (double)(1u << MAX_LEVEL) * (1.0 / (hi - lo));
    int ix           = (int)(floor(x * m) - lo * m);
    return (unsigned)(ix < mcoord ? ix : mcoord);
}

void orc_sfc_keys(size_t n, const double* x, const double* y, const double* z, const orc_box* b, uint64_t* keys)
{
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        if (keys[i] == REMOVE_KEY) { continue; }
        keys[i] = orc_hilbert(quantise(x[i], b->lo[0], b->hi[0]), quantise(y[i], b->lo[1], b->hi[1]),
                              quantise(z[i], b->lo[2], b->hi[2]));
    }
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* stable key sort: the permutation of std::stable_sort on (key, index) (cstone/primitives/gather.hpp:42-67)          */
/* ---------------------------------------------------------------------------------------------------------------- */

typedef struct
{
    uint64_t key;
    uint32_t idx;
} KeyIdx;

static int cmpKeyIdx(const void* a, const void* b)
{
    const KeyIdx* p = (const KeyIdx*)a;
    const KeyIdx* q = (const KeyIdx*)b;
    if (p->key != q->key) { return p->key < q->key ? -1 : 1; }
    return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

void orc_sort_by_key(size_t n, uint64_t* keys, uint32_t* perm)
{
    KeyIdx* t = (KeyIdx*)malloc(n * sizeof(KeyIdx));
    for (size_t i = 0; i < n; ++i)
    {
        t[i].key = keys[i];
        t[i].idx = perm ? perm[i] : (uint32_t)i;
    }
    qsort(t, n, sizeof(KeyIdx), cmpKeyIdx);
    for (size_t i = 0; i < n; ++i)
    {
        keys[i] = t[i].key;
        if (perm) { perm[i] = t[i].idx; }
    }
    free(t);
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* cornerstone leaf tree: cstone/tree/csarray.hpp:76-86 (counts), 248-290 (node ops), 340-389 (rebalance),            */
/* 409-440 (updateOctree / computeOctree)                                                                            */
/* ---------------------------------------------------------------------------------------------------------------- */

static size_t lowerBound(const uint64_t* a, size_t n, uint64_t v)
{
    size_t lo = 0, hi = n;
    while (lo < hi)
    {
        size_t mid = (lo + hi) / 2;
        if (a[mid] < v) { lo = mid + 1; }
        else { hi = mid; }
    }
    return lo;
}

static unsigned levelOfRange(uint64_t range) { return (unsigned)__builtin_clzll(range) / 3u; }
static uint64_t rangeOfLevel(unsigned level) { return UINT64_C(1) << (3u * (MAX_LEVEL - level)); }

static void leafCounts(const uint64_t* leaves, size_t L, const uint64_t* keys, size_t n, unsigned* counts)
{
    for (size_t i = 0; i < L; ++i)
    {
        counts[i] = (unsigned)(lowerBound(keys, n, leaves[i + 1]) - lowerBound(keys, n, leaves[i]));
    }
}

static int nodeOp(const uint64_t* leaves, size_t i, const unsigned* counts, unsigned bucket)
{
    uint64_t key   = leaves[i];
    unsigned level = levelOfRange(leaves[i + 1] - key);
    if (level > 0)
    {
        int sib = (int)((key >> (3u * (MAX_LEVEL - level))) & 7u);
        if (sib > 0 && leaves[i - sib + 8] == leaves[i - sib] + rangeOfLevel(level - 1))
        {
            size_t parentCount = 0;
            for (int k = 0; k < 8; ++k)
            {
                parentCount += counts[i - sib + k];
            }
            if (parentCount <= bucket) { return 0; }
        }
    }
    unsigned c = counts[i];
    if (c > bucket * 512u && level + 3 < MAX_LEVEL) { return 4096; }
    if (c > bucket * 64u && level + 2 < MAX_LEVEL) { return 512; }
    if (c > bucket * 8u && level + 1 < MAX_LEVEL) { return 64; }
    if (c > bucket && level < MAX_LEVEL) { return 8; }
    return 1;
}

size_t orc_compute_octree(size_t n, const uint64_t* keys, unsigned bucket, uint64_t* leavesOut, unsigned* countsOut,
                          size_t cap)
{
    size_t L          = 1;
    uint64_t* leaves  = (uint64_t*)malloc(2 * sizeof(uint64_t));
    unsigned* counts  = (unsigned*)malloc(sizeof(unsigned));
    leaves[0]         = 0;
    leaves[1]         = ROOT_RANGE;
    counts[0]         = (unsigned)n;
    for (;;)
    {
        int* ops      = (int*)malloc((L + 1) * sizeof(int));
        int converged = 1;
        for (size_t i = 0; i < L; ++i)
        {
            ops[i] = nodeOp(leaves, i, counts, bucket);
            if (ops[i] != 1) { converged = 0; }
        }
        size_t newL = 0;
        for (size_t i = 0; i < L; ++i)
        {
            newL += (size_t)ops[i];
        }
        uint64_t* nl = (uint64_t*)malloc((newL + 1) * sizeof(uint64_t));
        size_t out   = 0;
        for (size_t i = 0; i < L; ++i)
        {
            unsigned level = levelOfRange(leaves[i + 1] - leaves[i]);
            if (ops[i] == 1) { nl[out++] = leaves[i]; }
            else if (ops[i] > 1)
            {
                unsigned diff = ops[i] == 8 ? 1 : ops[i] == 64 ? 2 : ops[i] == 512 ? 3 : 4;
                for (int s = 0; s < ops[i]; ++s)
                {
                    nl[out++] = leaves[i] + (uint64_t)s * rangeOfLevel(level + diff);
                }
            }
        }
        nl[newL] = ROOT_RANGE;
        free(ops);
        free(leaves);
        leaves = nl;
        L      = newL;
        free(counts);
        counts = (unsigned*)malloc(L * sizeof(unsigned));
        leafCounts(leaves, L, keys, n, counts);
        if (converged) { break; }
    }
    if (L + 1 <= cap)
    {
        memcpy(leavesOut, leaves, (L + 1) * sizeof(uint64_t));
        memcpy(countsOut, counts, L * sizeof(unsigned));
    }
    free(leaves);
    free(counts);
    return L;
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* kernel tables: sph/include/sph/kernels.hpp:36-59, sph/include/sph/sph_kernel_tables.hpp:22-102                    */
/* ---------------------------------------------------------------------------------------------------------------- */

static double sincH(double v)
{
    if (v == 0.0) { return 1.0; }
    double a = M_PI_2 * v;
    return sin(a) / a;
}

static double sincHDeriv(double v)
{
    if (v == 0.0) { return 0.0; }
    double a = M_PI_2 * v;
    double s = sin(a) / a;
    return s * M_PI_2 * ((cos(a) / sin(a)) - 1.0 / a);
}

static int cmpDouble(const void* a, const void* b)
{
    double p = *(const double*)a, q = *(const double*)b;
    return p < q ? -1 : (p > q);
}

double orc_kernel_tables(double n, double* wh, double* whd)
{
    const int N = 2000;
    double h    = 2.0 / N;
    double odd[1000], even[999];
    for (int i = 0; i < 1000; ++i)
    {
        double x = (2 * (i + 1) - 1) * h;
        odd[i]   = 4.0 * M_PI * x * x * pow(sincH(x), n);
    }
    for (int i = 0; i < 999; ++i)
    {
        double x = (2 * (i + 1)) * h;
        even[i]  = 4.0 * M_PI * x * x * pow(sincH(x), n);
    }
    qsort(odd, 1000, sizeof(double), cmpDouble);
    qsort(even, 999, sizeof(double), cmpDouble);
    double so = 0.0, se = 0.0;
    for (int i = 0; i < 1000; ++i)
    {
        so += odd[i];
    }
    for (int i = 0; i < 999; ++i)
    {
        se += even[i];
    }
    double fa = 0.0, fb = 4.0 * M_PI * 2.0 * 2.0 * pow(sincH(2.0), n);
    double K  = 1.0 / (h / 3.0 * (fa + fb + 4.0 * so + 2.0 * se));
    double dx = 2.0 / (ORC_TABLE - 1);
    for (int i = 0; i < ORC_TABLE; ++i)
    {
        double x = 0.0 + i * dx;
        wh[i]    = pow(sincH(x), n);
        whd[i]   = n * pow(sincH(x), n - 1) * sincHDeriv(x);
    }
    return K;
}

double orc_sphynx_3d_k(double n)
{
    double b0 = 2.7012593e-2, b1 = 2.0410827e-2, b2 = 3.7451957e-3, b3 = 4.7013839e-2;
    return b0 + b1 * sqrt(n) + b2 * n + b3 * sqrt(n * n * n);
}

/* sph/include/sph/table_lookup.hpp:14-26 */
static double lookup(const double* table, double v)
{
    const int numIntervals = ORC_TABLE - 1;
    const double dx        = 2.0 / numIntervals;
    const double invDx     = 1.0 / dx;
    int idx                = (int)(v * invDx);
    if (idx >= numIntervals) { return 0.0; }
    double derivative = (table[idx + 1] - table[idx]) * invDx;
    return table[idx] + derivative * (v - (double)idx * dx);
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* neighbour search: cstone/findneighbors.hpp:33-51,77-147 (exact test), sph/include/sph/find_neighbors.hpp:10-41    */
/* (smoothing-length iteration), sph/include/sph/kernels.hpp:27-33 (updateH). Lists ascending in j, first ngmax kept */
/* ---------------------------------------------------------------------------------------------------------------- */

static double updateH(unsigned ng0, unsigned nc, double h)
{
    return h * 0.5 * pow(1.0 + 1023.0 * ng0 / (double)nc, 0.1);
}

typedef struct
{
    int nc[3];
    double lo[3], cs[3];
    int* start; /* [cells+1] */
    int* idx;
} Grid;

static int cellCoord(double v, int k, const Grid* g)
{
    int c = (int)floor((v - g->lo[k]) / g->cs[k]);
    if (c < 0) { c = 0; }
    if (c >= g->nc[k]) { c = g->nc[k] - 1; }
    return c;
}

static void buildGrid(Grid* g, size_t n, const double* x, const double* y, const double* z, const orc_box* b,
                      double reach)
{
    const double* P[3] = {x, y, z};
    for (int k = 0; k < 3; ++k)
    {
        double lo = b->lo[k], hi = b->hi[k];
        if (!b->periodic[k])
        {
            for (size_t i = 0; i < n; ++i)
            {
                lo = P[k][i] < lo ? P[k][i] : lo;
                hi = P[k][i] > hi ? P[k][i] : hi;
            }
        }
        int nc   = (int)floor((hi - lo) / reach);
        nc       = nc < 1 ? 1 : (nc > 256 ? 256 : nc);
        g->nc[k] = nc;
        g->lo[k] = lo;
        g->cs[k] = (hi - lo) / nc;
    }
    size_t cells = (size_t)g->nc[0] * g->nc[1] * g->nc[2];
    g->start     = (int*)calloc(cells + 1, sizeof(int));
    g->idx       = (int*)malloc(n * sizeof(int));
    int* cellOf  = (int*)malloc(n * sizeof(int));
    for (size_t i = 0; i < n; ++i)
    {
        int c     = (cellCoord(z[i], 2, g) * g->nc[1] + cellCoord(y[i], 1, g)) * g->nc[0] + cellCoord(x[i], 0, g);
        cellOf[i] = c;
        g->start[c + 1]++;
    }
    for (size_t c = 0; c < cells; ++c)
    {
        g->start[c + 1] += g->start[c];
    }
    int* fill = (int*)calloc(cells, sizeof(int));
    for (size_t i = 0; i < n; ++i)
    {
        g->idx[g->start[cellOf[i]] + fill[cellOf[i]]++] = (int)i;
    }
    free(fill);
    free(cellOf);
}

static int cmpU32(const void* a, const void* b)
{
    uint32_t p = *(const uint32_t*)a, q = *(const uint32_t*)b;
    return p < q ? -1 : (p > q);
}

/* count (and store, ascending, at most ngmax) the neighbours of i within 2 h_i */
static unsigned searchOne(size_t i, size_t n, const double* x, const double* y, const double* z, double hi,
                          const orc_box* b, const Grid* g, unsigned ngmax, uint32_t* out, uint32_t* tmp, size_t tmpCap)
{
    double L[3], iL[3];
    for (int k = 0; k < 3; ++k)
    {
        L[k]  = b->hi[k] - b->lo[k];
        iL[k] = 1.0 / L[k];
    }
    double radiusSq = 4.0 * hi * hi;
    size_t found    = 0;
    int brute       = 0;
    for (int k = 0; k < 3; ++k)
    {
        if (2.0 * hi > g->cs[k] && g->nc[k] > 1) { brute = 1; }
    }
    int span[3], c0[3];
    const double* P[3] = {x, y, z};
    for (int k = 0; k < 3; ++k)
    {
        c0[k]   = cellCoord(P[k][i], k, g);
        span[k] = (g->nc[k] < 3 || brute) ? g->nc[k] : 3;
    }
    for (int a = 0; a < span[2]; ++a)
    {
        for (int bb = 0; bb < span[1]; ++bb)
        {
            for (int c = 0; c < span[0]; ++c)
            {
                int cc[3], ok = 1;
                int off[3] = {c, bb, a};
                for (int k = 0; k < 3; ++k)
                {
                    if (span[k] == g->nc[k]) { cc[k] = off[k]; }
                    else
                    {
                        cc[k] = c0[k] + off[k] - 1;
                        if (cc[k] < 0 || cc[k] >= g->nc[k])
                        {
                            if (b->periodic[k]) { cc[k] = (cc[k] + g->nc[k]) % g->nc[k]; }
                            else { ok = 0; }
                        }
                    }
                }
                if (!ok) { continue; }
                int cell = (cc[2] * g->nc[1] + cc[1]) * g->nc[0] + cc[0];
                for (int s = g->start[cell]; s < g->start[cell + 1]; ++s)
                {
                    size_t j = (size_t)g->idx[s];
                    if (j == i) { continue; }
                    double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
                    if (b->periodic[0]) { dx -= L[0] * rint(dx * iL[0]); }
                    if (b->periodic[1]) { dy -= L[1] * rint(dy * iL[1]); }
                    if (b->periodic[2]) { dz -= L[2] * rint(dz * iL[2]); }
                    if (dx * dx + dy * dy + dz * dz < radiusSq)
                    {
                        if (found < tmpCap) { tmp[found] = (uint32_t)j; }
                        found++;
                    }
                }
            }
        }
    }
    (void)n;
    size_t keep = found < tmpCap ? found : tmpCap;
    qsort(tmp, keep, sizeof(uint32_t), cmpU32);
    size_t store = keep < ngmax ? keep : ngmax;
    if (out) { memcpy(out, tmp, store * sizeof(uint32_t)); }
    return (unsigned)found;
}

void orc_find_neighbors(size_t n, const double* x, const double* y, const double* z, double* h, const orc_box* b,
                        unsigned ng0, unsigned ngmax, int iterate, uint32_t* nbr, unsigned* nc)
{
    double hmax = 0.0;
    for (size_t i = 0; i < n; ++i)
    {
        hmax = h[i] > hmax ? h[i] : hmax;
    }
    Grid g;
    buildGrid(&g, n, x, y, z, b, 2.0 * hmax);
    unsigned ngmin = ng0 / 4;
#pragma omp parallel
    {
        size_t cap    = n;
        uint32_t* tmp = (uint32_t*)malloc(cap * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 64)
        for (size_t i = 0; i < n; ++i)
        {
            unsigned ncSph = 1 + searchOne(i, n, x, y, z, h[i], b, &g, ngmax, nbr + i * ngmax, tmp, cap);
            int it         = 0;
            while (iterate && (ngmin > ncSph || (ncSph - 1) > ngmax) && it++ < 10)
            {
                h[i]  = updateH(ng0, ncSph, h[i]);
                ncSph = 1 + searchOne(i, n, x, y, z, h[i], b, &g, ngmax, nbr + i * ngmax, tmp, cap);
            }
            nc[i] = ncSph;
        }
        free(tmp);
    }
    free(g.start);
    free(g.idx);
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* J-loops (FP64)                                                                                                    */
/* ---------------------------------------------------------------------------------------------------------------- */

/* legacy periodic shift, cstone/sfc/box.hpp applyPBC: by one box length if the component exceeds r */
static void pbcShift(const orc_box* b, double r, double* xx, double* yy, double* zz)
{
    double* c[3] = {xx, yy, zz};
    for (int k = 0; k < 3; ++k)
    {
        if (!b->periodic[k]) { continue; }
        double L = b->hi[k] - b->lo[k];
        if (*c[k] > r) { *c[k] -= L; }
        else if (*c[k] < -r) { *c[k] += L; }
    }
}

/* sph/include/sph/hydro_ve/xmass_kern.hpp:50-79 */
double orc_xmass(unsigned i, double K, const orc_box* b, const uint32_t* nb, unsigned cnt, const double* x,
                 const double* y, const double* z, const double* h, const double* m, const double* wh)
{
    double hi = h[i], mi = m[i];
    double hInv = 1.0 / hi, h3Inv = hInv * hInv * hInv;
    double rho0 = mi;
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double xx = x[i] - x[j], yy = y[i] - y[j], zz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &xx, &yy, &zz);
        double dist = sqrt(xx * xx + yy * yy + zz * zz);
        rho0 += lookup(wh, dist * hInv) * m[j];
    }
    return mi / (rho0 * K * h3Inv);
}

/* sph/include/sph/hydro_ve/ve_def_gradh_kern.hpp:43-90 */
void orc_ve_def_gradh(unsigned i, double K, const orc_box* b, const uint32_t* nb, unsigned cnt, const double* x,
                      const double* y, const double* z, const double* h, const double* m, const double* wh,
                      const double* whd, const double* xm, double* kxOut, double* gradhOut)
{
    double hi = h[i], mi = m[i], xmassi = xm[i];
    double hInv = 1.0 / hi, h3Inv = hInv * hInv * hInv;
    double kxi = xmassi, whomegai = -3.0 * xmassi, wrho0i = -3.0 * mi;
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double xx = x[i] - x[j], yy = y[i] - y[j], zz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &xx, &yy, &zz);
        double dist  = sqrt(xx * xx + yy * yy + zz * zz);
        double vloc  = dist * hInv;
        double w     = lookup(wh, vloc);
        double dw    = lookup(whd, vloc);
        double dterh = -(3.0 * w + vloc * dw);
        kxi += w * xm[j];
        whomegai += dterh * xm[j];
        wrho0i += dterh * m[j];
    }
    kxi *= K * h3Inv;
    whomegai *= K * h3Inv * hInv;
    wrho0i *= K * h3Inv * hInv;
    whomegai      = whomegai * mi / xmassi + (kxi - K * xmassi * h3Inv) * wrho0i;
    double rhoi   = kxi * mi / xmassi;
    double dhdrho = -hi / (rhoi * 3.0);
    *kxOut        = kxi;
    *gradhOut     = 1.0 - dhdrho * whomegai;
}

static int expOf(double v) { return v == 0.0 ? 0 : ilogb(v); }

/* sph/include/sph/hydro_ve/iad_kern.hpp:43-110 */
void orc_iad(unsigned i, double K, const orc_box* b, const uint32_t* nb, unsigned cnt, const double* x,
             const double* y, const double* z, const double* h, const double* wh, const double* xm, const double* kx,
             double c[6])
{
    double t11 = 0, t12 = 0, t13 = 0, t22 = 0, t23 = 0, t33 = 0;
    double hi = h[i], hiInv = 1.0 / hi;
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &rx, &ry, &rz);
        double dist  = sqrt(rx * rx + ry * ry + rz * rz);
        double w     = lookup(wh, dist * hiInv);
        double voljw = xm[j] / kx[j] * w;
        t11 += rx * rx * voljw;
        t12 += rx * ry * voljw;
        t13 += rx * rz * voljw;
        t22 += ry * ry * voljw;
        t23 += ry * rz * voljw;
        t33 += rz * rz * voljw;
    }
    int es      = expOf(t11) + expOf(t12) + expOf(t13) + expOf(t22) + expOf(t23) + expOf(t33);
    double norm = ldexp(1.0, -es / 6);
    t11 *= norm;
    t12 *= norm;
    t13 *= norm;
    t22 *= norm;
    t23 *= norm;
    t33 *= norm;
    double det = t11 * t22 * t33 + 2.0 * t12 * t23 * t13 - t11 * t23 * t23 - t22 * t13 * t13 - t33 * t12 * t12;
    double factor = norm * (hi * hi * hi) / (det * K);
    if (isnan(factor) && cnt == 0) { factor = 0.0; }
    c[0] = (t22 * t33 - t23 * t23) * factor;
    c[1] = (t13 * t23 - t33 * t12) * factor;
    c[2] = (t12 * t23 - t22 * t13) * factor;
    c[3] = (t11 * t33 - t13 * t13) * factor;
    c[4] = (t13 * t12 - t11 * t23) * factor;
    c[5] = (t11 * t22 - t12 * t12) * factor;
}

/* sph/include/sph/hydro_ve/divv_curlv_kern.hpp:43-123 */
void orc_divv_curlv(unsigned i, double K, const orc_box* b, const uint32_t* nb, unsigned cnt, const double* x,
                    const double* y, const double* z, const double* vx, const double* vy, const double* vz,
                    const double* h, const double* const cij[6], const double* wh, const double* kx,
                    const double* xm, double* divvOut, double* curlvOut, double dv[6])
{
    double hi = h[i], hiInv = 1.0 / hi, hiInv3 = hiInv * hiInv * hiInv;
    double dVx[3] = {0, 0, 0}, dVy[3] = {0, 0, 0}, dVz[3] = {0, 0, 0};
    double c11 = cij[0][i], c12 = cij[1][i], c13 = cij[2][i], c22 = cij[3][i], c23 = cij[4][i], c33 = cij[5][i];
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &rx, &ry, &rz);
        double r2   = rx * rx + ry * ry + rz * rz;
        double dist = sqrt(r2);
        double vxji = vx[j] - vx[i], vyji = vy[j] - vy[i], vzji = vz[j] - vz[i];
        double Wi   = lookup(wh, dist * hiInv);
        double tA[3];
        tA[0] = -(c11 * rx + c12 * ry + c13 * rz) * Wi;
        tA[1] = -(c12 * rx + c22 * ry + c23 * rz) * Wi;
        tA[2] = -(c13 * rx + c23 * ry + c33 * rz) * Wi;
        for (int k = 0; k < 3; ++k)
        {
            dVx[k] += (vxji * xm[j]) * tA[k];
            dVy[k] += (vyji * xm[j]) * tA[k];
            dVz[k] += (vzji * xm[j]) * tA[k];
        }
    }
    double nk = K * hiInv3 / kx[i];
    *divvOut  = nk * (dVx[0] + dVy[1] + dVz[2]);
    double cx = dVz[1] - dVy[2], cy = dVx[2] - dVz[0], cz = dVy[0] - dVx[1];
    *curlvOut = nk * sqrt(cx * cx + cy * cy + cz * cz);
    dv[0]     = nk * dVx[0];
    dv[1]     = nk * (dVx[1] + dVy[0]);
    dv[2]     = nk * (dVx[2] + dVz[0]);
    dv[3]     = nk * dVy[1];
    dv[4]     = nk * (dVy[2] + dVz[1]);
    dv[5]     = nk * dVz[2];
}

/* sph/include/sph/hydro_ve/av_switches_kern.hpp:43-137 */
double orc_av_switches(unsigned i, double K, const orc_box* b, const uint32_t* nb, unsigned cnt, const double* x,
                       const double* y, const double* z, const double* vx, const double* vy, const double* vz,
                       const double* h, const double* c, const double* const cij[6], const double* wh,
                       const double* kx, const double* xm, const double* divv, double dt, double alphamin,
                       double alphamax, double decay, double alpha_i)
{
    double hi = h[i], ci = c[i];
    double vsigI = 1.e-40 * ci;
    double hiInv = 1.0 / hi, hiInv3 = hiInv * hiInv * hiInv;
    double divvI = divv[i];
    double gx = 0, gy = 0, gz = 0;
    double c11 = cij[0][i], c12 = cij[1][i], c13 = cij[2][i], c22 = cij[3][i], c23 = cij[4][i], c33 = cij[5][i];
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &rx, &ry, &rz);
        double r2   = rx * rx + ry * ry + rz * rz;
        double dist = sqrt(r2);
        double vxij = vx[i] - vx[j], vyij = vy[i] - vy[j], vzij = vz[i] - vz[j];
        double rv   = rx * vxij + ry * vyij + rz * vzij;
        double vs   = 0.0;
        if (rv < 0.0) { vs = ci + c[j] - 3.0 * rv / dist; }
        vsigI       = vsigI > vs ? vsigI : vs;
        double Wi   = K * hiInv3 * lookup(wh, dist * hiInv);
        double tA1  = -(c11 * rx + c12 * ry + c13 * rz) * Wi;
        double tA2  = -(c12 * rx + c22 * ry + c23 * rz) * Wi;
        double tA3  = -(c13 * rx + c23 * ry + c33 * rz) * Wi;
        double fac  = xm[j] / kx[j] * (divvI - divv[j]);
        gx += fac * tA1;
        gy += fac * tA2;
        gz += fac * tA3;
    }
    double graddivv = sqrt(gx * gx + gy * gy + gz * gz);
    double alphaloc = 0.0;
    if (divvI < 0.0)
    {
        double aConst = hi * hi * graddivv;
        alphaloc      = alphamax * aConst / (aConst + hi * fabs(divvI) + 0.05 * ci);
    }
    if (alphaloc >= alpha_i) { return alphaloc; }
    double dec  = hi / (decay * vsigI);
    double adot = alphaloc >= alphamin ? (alphaloc - alpha_i) / dec : (alphamin - alpha_i) / dec;
    return alpha_i + adot * dt;
}

/* sph/include/sph/hydro_ve/momentum_energy_kern.hpp:43-222; artificial_viscosity sph/include/sph/kernels.hpp:71-85.
 * out: ax, ay, az, du, maxvsignal */
void orc_momentum_energy(unsigned i, int avClean, double K, const orc_box* b, const uint32_t* nb, unsigned cnt,
                         const double* x, const double* y, const double* z, const double* vx, const double* vy,
                         const double* vz, const double* h, const double* m, const double* prho, const double* c,
                         const double* const cij[6], double Atmin, double Atmax, double ramp, const double* wh,
                         const double* kx, const double* xm, const double* alpha, const double* const dv[6],
                         double out[5])
{
    double hi = h[i], mi = m[i], ci = c[i], kxi = kx[i], alphai = alpha[i], xmassi = xm[i];
    double rhoi = kxi * mi / xmassi, prhoi = prho[i];
    double hiInv = 1.0 / hi, hiInv3 = hiInv * hiInv * hiInv;
    double maxvs = 0.0, mx = 0.0, my = 0.0, mz = 0.0, energy = 0.0, aViscE = 0.0;
    double c11 = cij[0][i], c12 = cij[1][i], c13 = cij[2][i], c22 = cij[3][i], c23 = cij[4][i], c33 = cij[5][i];
    double gi[6] = {0, 0, 0, 0, 0, 0};
    if (avClean)
    {
        for (int k = 0; k < 6; ++k)
        {
            gi[k] = dv[k][i];
        }
    }
    double etaCrit = cbrt(32.0 * M_PI / 3.0 / (double)(cnt + 1));
    for (unsigned q = 0; q < cnt; ++q)
    {
        uint32_t j = nb[q];
        double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        pbcShift(b, 2.0 * hi, &rx, &ry, &rz);
        double r2   = rx * rx + ry * ry + rz * rz;
        double dist = sqrt(r2);
        double vxij = vx[i] - vx[j], vyij = vy[i] - vy[j], vzij = vz[i] - vz[j];
        double hj = h[j], hjInv = 1.0 / hj;
        double v1 = dist * hiInv, v2 = dist * hjInv;
        double hjInv3 = hjInv * hjInv * hjInv;
        double Wi = hiInv3 * lookup(wh, v1), Wj = hjInv3 * lookup(wh, v2);
        double tA1i = -(c11 * rx + c12 * ry + c13 * rz) * Wi;
        double tA2i = -(c12 * rx + c22 * ry + c23 * rz) * Wi;
        double tA3i = -(c13 * rx + c23 * ry + c33 * rz) * Wi;
        double d11 = cij[0][j], d12 = cij[1][j], d13 = cij[2][j], d22 = cij[3][j], d23 = cij[4][j], d33 = cij[5][j];
        double tA1j = -(d11 * rx + d12 * ry + d13 * rz) * Wj;
        double tA2j = -(d12 * rx + d22 * ry + d23 * rz) * Wj;
        double tA3j = -(d13 * rx + d23 * ry + d33 * rz) * Wj;
        double mj = m[j], cj = c[j], xmassj = xm[j];
        double rhoj = kx[j] * mj / xmassj;
        double rv   = rx * vxij + ry * vyij + rz * vzij;
        if (avClean)
        {
            /* avRvCorrection, momentum_energy_kern.hpp:43-63 */
            double R[3]  = {rx, ry, rz};
            double gj[6] = {dv[0][j], dv[1][j], dv[2][j], dv[3][j], dv[4][j], dv[5][j]};
            double si[3] = {gi[0] * R[0] + gi[1] * R[1] + gi[2] * R[2], gi[3] * R[1] + gi[4] * R[2], gi[5] * R[2]};
            double sj[3] = {gj[0] * R[0] + gj[1] * R[1] + gj[2] * R[2], gj[3] * R[1] + gj[4] * R[2], gj[5] * R[2]};
            double d1 = R[0] * si[0] + R[1] * si[1] + R[2] * si[2];
            double d2 = R[0] * sj[0] + R[1] * sj[1] + R[2] * sj[2];
            double d3 = 1.0, eta = v1 < v2 ? v1 : v2;
            if (eta < etaCrit)
            {
                double e = 5.0 * (eta - etaCrit);
                d3       = exp(-e * e);
            }
            double A   = d2 != 0.0 ? d1 / d2 : 0.0;
            double Ap1 = 1.0 + A;
            double lim = 4.0 * A / (Ap1 * Ap1);
            lim        = lim < 1.0 ? lim : 1.0;
            lim        = lim > 0.0 ? lim : 0.0;
            rv += -(0.5 * d3 * lim) * (d1 + d2);
        }
        double wij  = rv / dist;
        double visc = 0.0;
        if (wij < 0.0)
        {
            double vsig = (alphai + alpha[j]) * 0.25 * (ci + cj) - 2.0 * wij;
            visc        = -vsig * wij;
        }
        double vijs = 0.5 * (ci + cj) - 2.0 * wij;
        maxvs       = vijs > maxvs ? vijs : maxvs;
        double aMom, bMom;
        double atw = fabs(rhoi - rhoj) / (rhoi + rhoj);
        if (atw < Atmin)
        {
            aMom = xmassi * xmassi;
            bMom = xmassj * xmassj;
        }
        else if (atw > Atmax)
        {
            aMom = xmassi * xmassj;
            bMom = aMom;
        }
        else
        {
            double s = ramp * (atw - Atmin);
            aMom     = pow(xmassi, 2.0 - s) * pow(xmassj, s);
            bMom     = pow(xmassj, 2.0 - s) * pow(xmassi, s);
        }
        double aVisc = mj / rhoi * visc, bVisc = mj / rhoj * visc;
        double avx = 0.5 * (aVisc * tA1i + bVisc * tA1j);
        double avy = 0.5 * (aVisc * tA2i + bVisc * tA2j);
        double avz = 0.5 * (aVisc * tA3i + bVisc * tA3j);
        aViscE += avx * vxij + avy * vyij + avz * vzij;
        energy += mj * aMom * (vxij * tA1i + vyij * tA2i + vzij * tA3i);
        double momI = mj * prhoi * aMom, momJ = mj * prho[j] * bMom;
        mx += momI * tA1i + momJ * tA1j + avx;
        my += momI * tA2i + momJ * tA2j + avy;
        mz += momI * tA3i + momJ * tA3j + avz;
    }
    aViscE = aViscE > 0.0 ? aViscE : 0.0;
    out[3] = K * (prhoi * energy + 0.5 * aViscE);
    out[0] = -K * mx;
    out[1] = -K * my;
    out[2] = -K * mz;
    out[4] = maxvs;
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* whole step at one rank: main/src/propagator/ve_hydro.hpp:126-220                                                  */
/* ---------------------------------------------------------------------------------------------------------------- */

enum
{
    F_X, F_Y, F_Z, F_H, F_M, F_TEMP, F_VX, F_VY, F_VZ, F_XM1, F_YM1, F_ZM1, F_DUM1, F_ALPHA, NUM_CONS
};
static const char* const consNames[NUM_CONS] = {"x",  "y",  "z",    "h",    "m",    "temp",  "vx",
                                                "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha"};
enum
{
    D_XM, D_KX, D_GRADH, D_PRHO, D_C, D_C11, D_C12, D_C13, D_C22, D_C23, D_C33, D_DIVV, D_CURLV, D_AX, D_AY, D_AZ,
    D_DU, D_NC, D_DV11, D_DV12, D_DV13, D_DV22, D_DV23, D_DV33, NUM_DEP
};
static const char* const depNames[NUM_DEP] = {"xm",   "kx",   "gradh", "prho", "c",    "c11",   "c12", "c13",
                                              "c22",  "c23",  "c33",   "divv", "curlv", "ax",   "ay",  "az",
                                              "du",   "nc",   "dV11",  "dV12", "dV13",  "dV22", "dV23", "dV33"};

struct orc_sim
{
    size_t n;
    double* f[NUM_CONS];
    double* d[NUM_DEP];
    uint64_t* id;
    uint64_t* keys;
    uint32_t* nbr;
    orc_box box;
    int firstBox;
    unsigned ng0, ngmax;
    double gamma, mui, Kcour, Krho, alphamin, alphamax, decay;
    double minDt, minDt_m1, minDtCourant, minDtRho, ttot;
    double etot, ecin, eint, linmom, angmom, totalNeighbors;
    double iteration;
    int avClean; /* HydroVeProp<avClean = true>: IAD keeps the velocity gradients, MomentumEnergy corrects r.v */
    double K;
    double wh[ORC_TABLE], whd[ORC_TABLE];
};

orc_sim* orc_sim_create(size_t n, const double* const* fields, const uint64_t* id, const double* lim, int periodic,
                        const double* prm)
{
    orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
    s->n       = n;
    for (int k = 0; k < NUM_CONS; ++k)
    {
        s->f[k] = (double*)malloc(n * sizeof(double));
        memcpy(s->f[k], fields[k], n * sizeof(double));
    }
    for (int k = 0; k < NUM_DEP; ++k)
    {
        s->d[k] = (double*)calloc(n, sizeof(double));
    }
    s->id   = (uint64_t*)malloc(n * sizeof(uint64_t));
    s->keys = (uint64_t*)calloc(n, sizeof(uint64_t));
    memcpy(s->id, id, n * sizeof(uint64_t));
    for (int k = 0; k < 3; ++k)
    {
        s->box.lo[k]       = lim[2 * k];
        s->box.hi[k]       = lim[2 * k + 1];
        s->box.periodic[k] = periodic;
    }
    s->firstBox  = 1;
    s->ng0       = (unsigned)prm[0];
    s->ngmax     = (unsigned)prm[1];
    s->gamma     = prm[2];
    s->mui       = prm[3];
    s->minDt     = prm[4];
    s->minDt_m1  = prm[5];
    s->Kcour     = prm[6];
    s->Krho      = prm[7];
    s->alphamin  = prm[8];
    s->alphamax  = prm[9];
    s->decay     = prm[10];
    s->iteration = 1;
    s->nbr       = (uint32_t*)calloc(n * s->ngmax, sizeof(uint32_t));
    s->K         = orc_kernel_tables(6.0, s->wh, s->whd);
    return s;
}

void orc_sim_destroy(orc_sim* s)
{
    if (!s) { return; }
    for (int k = 0; k < NUM_CONS; ++k)
    {
        free(s->f[k]);
    }
    for (int k = 0; k < NUM_DEP; ++k)
    {
        free(s->d[k]);
    }
    free(s->id);
    free(s->keys);
    free(s->nbr);
    free(s);
}

/* box of open axes (cstone/sfc/box_mpi.hpp:69-107, box.hpp:398-414), keys, stable sort, reorder every field;
 * permOut (optional, n entries) receives the applied permutation (new index i held old index permOut[i]) */
void orc_sim_sync_perm(orc_sim* s, uint32_t* permOut)
{
    size_t n = s->n;
    for (int k = 0; k < 3; ++k)
    {
        if (s->box.periodic[k]) { continue; }
        double lo = INFINITY, hi = -INFINITY;
        for (size_t i = 0; i < n; ++i)
        {
            double v = s->f[F_X + k][i];
            lo       = v < lo ? v : lo;
            hi       = v > hi ? v : hi;
        }
        if (!s->firstBox)
        {
            double L  = s->box.hi[k] - s->box.lo[k];
            double l1 = s->box.lo[k] + 0.05 * L, h1 = s->box.hi[k] - 0.05 * L;
            lo        = lo < l1 ? lo : l1;
            hi        = hi > h1 ? hi : h1;
        }
        s->box.lo[k] = lo;
        s->box.hi[k] = hi;
    }
    s->firstBox = 0;
    orc_sfc_keys(n, s->f[F_X], s->f[F_Y], s->f[F_Z], &s->box, s->keys);
    uint32_t* perm = (uint32_t*)malloc(n * sizeof(uint32_t));
    for (size_t i = 0; i < n; ++i)
    {
        perm[i] = (uint32_t)i;
    }
    orc_sort_by_key(n, s->keys, perm);
    double* tmp = (double*)malloc(n * sizeof(double));
    for (int k = 0; k < NUM_CONS; ++k)
    {
        for (size_t i = 0; i < n; ++i)
        {
            tmp[i] = s->f[k][perm[i]];
        }
        memcpy(s->f[k], tmp, n * sizeof(double));
    }
    uint64_t* tid = (uint64_t*)malloc(n * sizeof(uint64_t));
    for (size_t i = 0; i < n; ++i)
    {
        tid[i] = s->id[perm[i]];
    }
    memcpy(s->id, tid, n * sizeof(uint64_t));
    if (permOut) { memcpy(permOut, perm, n * sizeof(uint32_t)); }
    free(tid);
    free(tmp);
    free(perm);
}

void orc_sim_sync(orc_sim* s) { orc_sim_sync_perm(s, NULL); }

static double idealCv(double mui, double gamma) { return 8.317e7 / mui / (gamma - 1.0); }

/* the force computation of HydroVeProp (ve_hydro.hpp:126-203); with an active mask, that of HydroVeBdtProp
 * (main/src/propagator/ve_hydro_bdt.hpp:224-296): the search for every particle, the J-loops for the active ones,
 * the EOS for every particle; avDt is the time step of the AV-switch update; dtOut (optional) receives the Courant
 * step of every active particle (INFINITY for the others) */
static int computeForcesImpl(orc_sim* s, const uint8_t* active, double avDt, double* dtOut)
{
    size_t n = s->n;
    double* x = s->f[F_X];
    double* y = s->f[F_Y];
    double* z = s->f[F_Z];
    double* h = s->f[F_H];
    unsigned* nc = (unsigned*)malloc(n * sizeof(unsigned));
    orc_find_neighbors(n, x, y, z, h, &s->box, s->ng0, s->ngmax, 1, s->nbr, nc);
    for (size_t i = 0; i < n; ++i)
    {
        s->d[D_NC][i] = nc[i];
    }
    const double* m = s->f[F_M];
    const double* cij[6] = {s->d[D_C11], s->d[D_C12], s->d[D_C13], s->d[D_C22], s->d[D_C23], s->d[D_C33]};
    const double* dv[6]  = {s->d[D_DV11], s->d[D_DV12], s->d[D_DV13], s->d[D_DV22], s->d[D_DV23], s->d[D_DV33]};
    double cv            = idealCv(s->mui, s->gamma);
    unsigned ng          = s->ngmax;
#define CNT(i) (nc[i] - 1 < ng ? nc[i] - 1 : ng)
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i]) { continue; }
        s->d[D_XM][i] = orc_xmass((unsigned)i, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, h, m, s->wh);
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i]) { continue; }
        orc_ve_def_gradh((unsigned)i, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, h, m, s->wh, s->whd,
                         s->d[D_XM], &s->d[D_KX][i], &s->d[D_GRADH][i]);
    }
    /* ideal-gas EOS with temp (sph/include/sph/hydro_ve/eos.hpp:52-94, sph/include/sph/eos.hpp:19-50) */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        double rho  = s->d[D_KX][i] * m[i] / s->d[D_XM][i];
        double tmpv = cv * s->f[F_TEMP][i] * (s->gamma - 1.0);
        double p    = rho * tmpv;
        s->d[D_C][i]    = sqrt(s->gamma * tmpv);
        s->d[D_PRHO][i] = p / (s->d[D_KX][i] * m[i] * m[i] * s->d[D_GRADH][i]);
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i]) { continue; }
        double c6[6];
        orc_iad((unsigned)i, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, h, s->wh, s->d[D_XM], s->d[D_KX], c6);
        for (int k = 0; k < 6; ++k)
        {
            s->d[D_C11 + k][i] = c6[k];
        }
    }
    double maxDivv = -INFINITY;
#pragma omp parallel for schedule(static) reduction(max : maxDivv)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i]) { continue; }
        double dvv[6];
        orc_divv_curlv((unsigned)i, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, s->f[F_VX], s->f[F_VY],
                       s->f[F_VZ], h, cij, s->wh, s->d[D_KX], s->d[D_XM], &s->d[D_DIVV][i], &s->d[D_CURLV][i], dvv);
        for (int k = 0; k < 6; ++k)
        {
            s->d[D_DV11 + k][i] = dvv[k];
        }
        maxDivv = s->d[D_DIVV][i] > maxDivv ? s->d[D_DIVV][i] : maxDivv;
    }
    /* rhoTimestep, sph/include/sph/ts_global.hpp:75-98 */
    s->minDtRho    = s->Krho / fabs(maxDivv);
    double* alphaN = (double*)malloc(n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i])
        {
            alphaN[i] = s->f[F_ALPHA][i];
            continue;
        }
        alphaN[i] = orc_av_switches((unsigned)i, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, s->f[F_VX],
                                    s->f[F_VY], s->f[F_VZ], h, s->d[D_C], cij, s->wh, s->d[D_KX], s->d[D_XM],
                                    s->d[D_DIVV], avDt, s->alphamin, s->alphamax, s->decay, s->f[F_ALPHA][i]);
    }
    memcpy(s->f[F_ALPHA], alphaN, n * sizeof(double));
    free(alphaN);
    double minDt = INFINITY;
    float kc     = (float)s->Kcour;
#pragma omp parallel for schedule(static) reduction(min : minDt)
    for (size_t i = 0; i < n; ++i)
    {
        if (active && !active[i])
        {
            if (dtOut) { dtOut[i] = INFINITY; }
            continue;
        }
        double o[5];
        orc_momentum_energy((unsigned)i, s->avClean, s->K, &s->box, s->nbr + i * ng, CNT(i), x, y, z, s->f[F_VX],
                            s->f[F_VY], s->f[F_VZ], h, m, s->d[D_PRHO], s->d[D_C], cij, 0.1, 0.2, 1.0 / (0.2 - 0.1),
                            s->wh, s->d[D_KX], s->d[D_XM], s->f[F_ALPHA], dv, o);
        s->d[D_AX][i] = o[0];
        s->d[D_AY][i] = o[1];
        s->d[D_AZ][i] = o[2];
        s->d[D_DU][i] = o[3];
        /* tsKCourant, sph/include/sph/kernels.hpp:10-17 (Kcour enters as float) */
        double v  = o[4] > 0.0 ? o[4] : s->d[D_C][i];
        double dt = h[i] > 0.0 ? (double)kc * h[i] / v : INFINITY;
        minDt     = dt < minDt ? dt : minDt;
        if (dtOut) { dtOut[i] = dt; }
    }
    s->minDtCourant = minDt;
#undef CNT
    /* conserved quantities, main/src/observables/conserved_quantities.hpp:48-175 */
    double ek = 0, ei = 0, p[3] = {0, 0, 0}, L[3] = {0, 0, 0}, ncs = 0;
    for (size_t i = 0; i < n; ++i)
    {
        double mi = m[i], X[3] = {x[i], y[i], z[i]}, V[3] = {s->f[F_VX][i], s->f[F_VY][i], s->f[F_VZ][i]};
        ek += mi * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
        ei += cv * s->f[F_TEMP][i] * mi;
        for (int k = 0; k < 3; ++k)
        {
            p[k] += mi * V[k];
        }
        L[0] += mi * (X[1] * V[2] - X[2] * V[1]);
        L[1] += mi * (X[2] * V[0] - X[0] * V[2]);
        L[2] += mi * (X[0] * V[1] - X[1] * V[0]);
        ncs += nc[i];
    }
    s->ecin           = 0.5 * ek;
    s->eint           = ei;
    s->etot           = s->ecin + s->eint;
    s->linmom         = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    s->angmom         = sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
    s->totalNeighbors = ncs;
    free(nc);
    return 0;
}

int orc_sim_compute_forces(orc_sim* s)
{
    orc_sim_sync(s);
    return computeForcesImpl(s, NULL, s->minDt, NULL);
}

void orc_sim_set_av_clean(orc_sim* s, int on) { s->avClean = on != 0; }

int orc_sim_forces_active(orc_sim* s, const uint8_t* active, double avDt, double* dtCourant)
{
    return computeForcesImpl(s, active, avDt, dtCourant);
}

/* positionUpdate of one axis (sph/include/sph/positions.hpp:100-111) */
static double pressAxis(double X, double A, double dX, double dt, double dtm1, double* V, double* dXn1)
{
    double vh = dX * (1.0 / dtm1);
    double vn = vh + 0.5 * dtm1 * A;
    *V        = vn + A * dt;
    *dXn1     = (vn + 0.5 * A * fabs(dt)) * dt;
    return X + *dXn1;
}

/* energyUpdate (positions.hpp:77-84) */
static double energyUpdate(double uOld, double dt, double dtm1, double du, double duM1)
{
    double uNew = uOld + du * dt + 0.5 * (du - duM1) / dtm1 * fabs(dt) * dt;
    if (uNew < 0.0) { uNew = uOld * exp(uNew * dt / uOld); }
    return uNew;
}

/* driftKernel (sph/include/sph/positions_gpu.cu:45-90) over the listed particles: back by dtBack, forward by dt from
 * there, no periodic folding */
void orc_drift(orc_sim* s, const uint32_t* idx, size_t cnt, float dt, float dtBack, const float* dtm1,
               const uint8_t* rung)
{
    double cv = idealCv(s->mui, s->gamma);
    for (size_t q = 0; q < cnt; ++q)
    {
        size_t i    = idx[q];
        double m1   = (double)dtm1[rung[i]];
        double back = -(double)dtBack, fwd = (double)dt;
        double A[3] = {s->d[D_AX][i], s->d[D_AY][i], s->d[D_AZ][i]};
        for (int k = 0; k < 3; ++k)
        {
            double v, d;
            double Xn          = pressAxis(s->f[F_X + k][i], A[k], s->f[F_XM1 + k][i], back, m1, &v, &d);
            s->f[F_X + k][i]   = pressAxis(Xn, A[k], s->f[F_XM1 + k][i], fwd, m1, &v, &d);
            s->f[F_VX + k][i]  = v;
        }
        double du = s->d[D_DU][i], duM1 = s->f[F_DUM1][i];
        double u  = energyUpdate(s->f[F_TEMP][i] * cv, back, m1, du, duM1);
        s->f[F_TEMP][i] = energyUpdate(u, fwd, m1, du, duM1) / cv;
    }
}

/* computePositionsKernel (positions_gpu.cu:117-166) over the listed particles; fold != 0: putInBox on the periodic
 * axes */
void orc_rung_positions(orc_sim* s, const uint32_t* idx, size_t cnt, float dt, const float* dtm1, const uint8_t* rung,
                        int fold)
{
    double cv = idealCv(s->mui, s->gamma);
    for (size_t q = 0; q < cnt; ++q)
    {
        size_t i    = idx[q];
        double m1   = (double)dtm1[rung[i]];
        double dtD  = (double)dt;
        double A[3] = {s->d[D_AX][i], s->d[D_AY][i], s->d[D_AZ][i]};
        for (int k = 0; k < 3; ++k)
        {
            double v, d;
            double X = pressAxis(s->f[F_X + k][i], A[k], s->f[F_XM1 + k][i], dtD, m1, &v, &d);
            if (fold && s->box.periodic[k])
            {
                double L = s->box.hi[k] - s->box.lo[k];
                if (X > s->box.hi[k]) { X -= L; }
                else if (X < s->box.lo[k]) { X += L; }
            }
            s->f[F_X + k][i]   = X;
            s->f[F_XM1 + k][i] = d;
            s->f[F_VX + k][i]  = v;
        }
        double du       = s->d[D_DU][i];
        s->f[F_TEMP][i] = energyUpdate(cv * s->f[F_TEMP][i], dtD, m1, du, s->f[F_DUM1][i]) / cv;
        s->f[F_DUM1][i] = du;
    }
}

/* updateSmoothingLength over the listed particles (sph/include/sph/update_h.hpp:12-47); returns 1 if any has
 * nc <= 1 */
int orc_update_h_subset(orc_sim* s, const uint32_t* idx, size_t cnt)
{
    int removed = 0;
    for (size_t q = 0; q < cnt; ++q)
    {
        size_t i     = idx[q];
        unsigned nci = (unsigned)s->d[D_NC][i];
        if (nci <= 1)
        {
            s->keys[i] = REMOVE_KEY;
            removed    = 1;
        }
        s->f[F_H][i] = updateH(s->ng0, nci, s->f[F_H][i]);
    }
    return removed;
}

/* computeTimestep (sph/include/sph/ts_global.hpp:100-128), positions + energy (sph/include/sph/positions.hpp:77-160),
 * smoothing-length update (sph/include/sph/update_h.hpp:12-33) */
int orc_sim_integrate(orc_sim* s)
{
    size_t n  = s->n;
    double dt = s->minDtCourant < s->minDtRho ? s->minDtCourant : s->minDtRho;
    double g  = 1.1 * s->minDt;
    dt        = dt < g ? dt : g;
    s->ttot += dt;
    s->minDt_m1 = s->minDt;
    s->minDt    = dt;
    double dtm1 = s->minDt_m1, adt = fabs(dt), cv = idealCv(s->mui, s->gamma);
    int removed = 0;
    for (size_t i = 0; i < n; ++i)
    {
        double A[3] = {s->d[D_AX][i], s->d[D_AY][i], s->d[D_AZ][i]};
        for (int k = 0; k < 3; ++k)
        {
            double dX   = s->f[F_XM1 + k][i];
            double vh   = dX * (1.0 / dtm1);
            double vn   = vh + 0.5 * dtm1 * A[k];
            double vnp1 = vn + A[k] * dt;
            double dXn  = (vn + 0.5 * A[k] * adt) * dt;
            double X    = s->f[F_X + k][i] + dXn;
            if (s->box.periodic[k])
            {
                double L = s->box.hi[k] - s->box.lo[k];
                if (X > s->box.hi[k]) { X -= L; }
                else if (X < s->box.lo[k]) { X += L; }
            }
            s->f[F_X + k][i]   = X;
            s->f[F_XM1 + k][i] = dXn;
            s->f[F_VX + k][i]  = vnp1;
        }
        double uOld = cv * s->f[F_TEMP][i], du = s->d[D_DU][i], duM1 = s->f[F_DUM1][i];
        double uNew = uOld + du * dt + 0.5 * (du - duM1) / dtm1 * adt * dt;
        if (uNew < 0.0) { uNew = uOld * exp(uNew * dt / uOld); }
        s->f[F_TEMP][i] = uNew / cv;
        s->f[F_DUM1][i] = du;
        unsigned nci    = (unsigned)s->d[D_NC][i];
        if (nci <= 1)
        {
            s->keys[i] = REMOVE_KEY;
            removed    = 1;
        }
        s->f[F_H][i] = updateH(s->ng0, nci, s->f[F_H][i]);
    }
    s->iteration += 1;
    return removed;
}

size_t orc_sim_size(const orc_sim* s) { return s->n; }

int orc_sim_get(const orc_sim* s, const char* name, double* out)
{
    for (int k = 0; k < NUM_CONS; ++k)
    {
        if (strcmp(name, consNames[k]) == 0)
        {
            memcpy(out, s->f[k], s->n * sizeof(double));
            return 0;
        }
    }
    for (int k = 0; k < NUM_DEP; ++k)
    {
        if (strcmp(name, depNames[k]) == 0)
        {
            memcpy(out, s->d[k], s->n * sizeof(double));
            return 0;
        }
    }
    if (strcmp(name, "id") == 0)
    {
        memcpy(out, s->id, s->n * sizeof(uint64_t));
        return 0;
    }
    return -1;
}

void orc_sim_keys(const orc_sim* s, uint64_t* out) { memcpy(out, s->keys, s->n * sizeof(uint64_t)); }

void orc_sim_neighbors(const orc_sim* s, uint32_t* out) { memcpy(out, s->nbr, s->n * s->ngmax * sizeof(uint32_t)); }

void orc_sim_scalars(const orc_sim* s, double* out)
{
    double v[18] = {s->minDt, s->minDt_m1, s->minDtCourant, s->minDtRho, s->ttot, s->etot, s->ecin, s->eint,
                    s->linmom, s->angmom, s->totalNeighbors, s->iteration, s->box.lo[0], s->box.hi[0],
                    s->box.lo[1], s->box.hi[1], s->box.lo[2], s->box.hi[2]};
    memcpy(out, v, sizeof(v));
}
