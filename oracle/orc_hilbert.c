/*
 * Compact Hilbert index, restated from src/hilbert.f90 (Hamilton's compact
 * Hilbert indices, Dalhousie TR CS-2006-07).  Test infrastructure only: the
 * oracle for the CUDA hot path.  Every helper keeps the reference's integer
 * semantics (3 dimensions, mask 7, d in {0,1,2}, level loop from the top).
 */
#include "rmpcd_oracle.h"

#define DIM 3
#define MASK 7

/* Fortran ibits(x, pos, 1) on a default (32-bit) integer */
static int bit1(int x, int pos) { return (int)(((unsigned)x >> pos) & 1u); }

/* rotate_right, src/hilbert.f90:20-29 */
static int rotate_right(int x, int d)
{
    unsigned ux = (unsigned)x;
    unsigned r = (ux >> d) | (ux << (DIM - d));
    return (int)(r & MASK);
}

/* rotate_left, src/hilbert.f90:31-40 */
static int rotate_left(int x, int d)
{
    unsigned ux = (unsigned)x;
    unsigned r = (ux << d) | (ux >> (DIM - d));
    return (int)(r & MASK);
}

/* gc, src/hilbert.f90:62-68 */
static int gc(int i) { return i ^ (int)((unsigned)i >> 1); }

/* entry_point, src/hilbert.f90:70-79 */
static int entry_point(int i) { return i == 0 ? 0 : gc(2 * ((i - 1) / 2)); }

/* inverse_gc, src/hilbert.f90:89-101 */
static int inverse_gc(int g)
{
    int r = g;
    for (int j = 1; j < DIM; j++) r ^= (int)((unsigned)g >> j);
    return r;
}

static int trailz(int x)
{
    if (x == 0) return 32;
    int n = 0;
    while (!((x >> n) & 1)) n++;
    return n;
}

/* intercube_g, src/hilbert.f90:103-109 */
static int intercube_g(int i) { return trailz(gc(i) ^ gc(i + 1)); }

static int fmodulo(int a, int p)
{
    int r = a % p;
    if (r != 0 && ((r < 0) != (p < 0))) r += p;
    return r;
}

/* intracube_d, src/hilbert.f90:111-122 */
static int intracube_d(int i)
{
    if (i == 0) return 0;
    if (fmodulo(i, 2) == 0) return fmodulo(intercube_g(i - 1), DIM);
    return fmodulo(intercube_g(i), DIM);
}

/* transform, src/hilbert.f90:124-129 */
static int transform(int e, int d, int b) { return rotate_right(b ^ e, d + 1); }

/* inverse_transform, src/hilbert.f90:131-137 */
static int inverse_transform(int e, int d, int b)
{
    return transform(rotate_right(e, d + 1), DIM - d - 2, b);
}

static int level_bits(const int p[3], int i)
{
    int l = 0;
    for (int j = 0; j < DIM; j++) l += (1 << j) * bit1(p[j], i);
    return l;
}

/* p_to_h, src/hilbert.f90:139-159 */
int orc_p_to_h(const int p[3], int m)
{
    int h = 0, e = 0, d = 2;
    for (int i = m - 1; i >= 0; i--) {
        int l = level_bits(p, i);
        l = transform(e, d, l);
        int w = inverse_gc(l);
        e = e ^ rotate_left(entry_point(w), d + 1);
        d = fmodulo(d + intracube_d(w) + 1, DIM);
        h = (int)((unsigned)h << DIM) | w;
    }
    return h;
}

/* h_to_p, src/hilbert.f90:161-186 */
void orc_h_to_p(int h, int m, int p[3])
{
    int e = 0, d = 2;
    p[0] = p[1] = p[2] = 0;
    for (int i = m - 1; i >= 0; i--) {
        int w = 0;
        for (int j = 0; j < DIM; j++) w += (1 << j) * bit1(h, i * DIM + j);
        int l = gc(w);
        l = inverse_transform(e, d, l);
        for (int j = 0; j < DIM; j++) p[j] += bit1(l, j) << i;
        e = e ^ rotate_left(entry_point(w), d + 1);
        d = fmodulo(d + intracube_d(w) + 1, DIM);
    }
}

/* gcr, src/hilbert.f90:188-200 */
static int gcr(int i, int mu)
{
    int r = 0;
    for (int k = DIM - 1; k >= 0; k--)
        if (bit1(mu, k) == 1) r = (int)((unsigned)r << 1) | bit1(i, k);
    return r;
}

/* inverse_gcr, src/hilbert.f90:202-223 */
static int inverse_gcr(int r, int mu, int pi)
{
    int i = 0, g = 0, j = -1;
    for (int k = 0; k < DIM; k++) j += bit1(mu, k);
    for (int k = DIM - 1; k >= 0; k--) {
        if (bit1(mu, k) == 1) {
            i |= bit1(r, j) << k;
            g |= fmodulo(bit1(i, k) + bit1(i, k + 1), 2) << k;
            j--;
        } else {
            g |= bit1(pi, k) << k;
            i |= fmodulo(bit1(g, k) + bit1(i, k + 1), 2) << k;
        }
    }
    return i;
}

/* extract_mask, src/hilbert.f90:225-239 */
static int extract_mask(int i, const int m[3])
{
    int mu = 0;
    for (int j = DIM - 1; j >= 0; j--) {
        mu = (int)((unsigned)mu << 1);
        if (m[j] > i) mu |= 1;
    }
    return mu;
}

static int popc3(int mu) { return bit1(mu, 0) + bit1(mu, 1) + bit1(mu, 2); }

static int maxval3(const int m[3])
{
    int r = m[0];
    if (m[1] > r) r = m[1];
    if (m[2] > r) r = m[2];
    return r;
}

/* compact_p_to_h, src/hilbert.f90:241-271 */
int orc_compact_p_to_h(const int p[3], const int m[3])
{
    int h = 0, e = 0, d = 2;
    int max_m = maxval3(m);
    for (int i = max_m - 1; i >= 0; i--) {
        int mu = extract_mask(i, m);
        int mu_norm = popc3(mu);
        mu = rotate_right(mu, d + 1);
        int l = level_bits(p, i);
        l = transform(e, d, l);
        int w = inverse_gc(l);
        int r = gcr(w, mu);
        e = e ^ rotate_left(entry_point(w), d + 1);
        d = fmodulo(d + intracube_d(w) + 1, DIM);
        h = (int)((unsigned)h << mu_norm) | r;
    }
    return h;
}

/* compact_h_to_p, src/hilbert.f90:273-307 */
void orc_compact_h_to_p(int h, const int m[3], int p[3])
{
    int e = 0, d = 2, k = 0;
    int max_m = maxval3(m);
    int sum_m = m[0] + m[1] + m[2];
    p[0] = p[1] = p[2] = 0;
    for (int i = max_m - 1; i >= 0; i--) {
        int mu = extract_mask(i, m);
        int mu_norm = popc3(mu);
        mu = rotate_right(mu, d + 1);
        int pi = rotate_right(e, d + 1) & (~mu & MASK);
        int r = 0;
        for (int j = 0; j < mu_norm; j++) r += (1 << j) * bit1(h, sum_m - k - mu_norm + j);
        k += mu_norm;
        int w = inverse_gcr(r, mu, pi);
        int l = gc(w);
        l = inverse_transform(e, d, l);
        for (int j = 0; j < DIM; j++) p[j] += bit1(l, j) << i;
        e = e ^ rotate_left(entry_point(w), d + 1);
        d = fmodulo(d + intracube_d(w) + 1, DIM);
    }
}
