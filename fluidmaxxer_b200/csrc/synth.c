/*
 * synth.c -- seeded synthetic geometries for the coupled LBM workloads.
 *
 * The reference reads its geometry from an ASCII VTI file (readVTI,
 * include/vti/VTIReader.hpp:35-160) and ships none; these generators produce
 * the solid masks of the benchmark problems from a seed, identically for the
 * CUDA path, the oracle and the CPU baseline.  Host-only, no CUDA.
 *
 * PRNG: splitmix64 seeding a xoshiro256** stream (Blackman & Vigna's published
 * generators); doubles are the top 53 bits scaled by 2^-53.
 * Cell index c = x + nx*(y + ny*z).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s[4]; } fm_rng;

static uint64_t splitmix64(uint64_t* x)
{
    uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

static void rng_seed(fm_rng* r, uint64_t seed)
{
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&x);
}

static uint64_t rng_next(fm_rng* r)
{
    uint64_t* s = r->s;
    const uint64_t out = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
}

static inline double rng_uniform(fm_rng* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }

/* n uniform doubles in [0,1) from `seed`. */
void fm_synth_uniform(uint64_t seed, long n, double* out)
{
    fm_rng r;
    rng_seed(&r, seed);
    for (long i = 0; i < n; ++i) out[i] = rng_uniform(&r);
}

static void apply_walls(int nx, int ny, int nz, uint8_t* m)
{
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            if (!(y == 0 || y == ny - 1 || z == 0 || z == nz - 1)) continue;
            uint8_t* row = m + (long)nx * (y + (long)ny * z);
            memset(row, 1, (size_t)nx);
        }
}

/* I.i.d. Bernoulli(p) solids: one draw per cell in index order; cells with
 * x < fluid_lo or x >= nx - fluid_hi are then forced fluid; with walls != 0
 * the y and z boundary layers become solid over the whole length. */
void fm_synth_bernoulli(int nx, int ny, int nz, double p, uint64_t seed, int fluid_lo,
                        int fluid_hi, int walls, uint8_t* mask)
{
    fm_rng r;
    rng_seed(&r, seed);
    const long n = (long)nx * ny * nz;
    for (long c = 0; c < n; ++c) {
        const int x = (int)(c % nx);
        const uint8_t s = rng_uniform(&r) < p;
        mask[c] = (x < fluid_lo || x >= nx - fluid_hi) ? 0 : s;
    }
    if (walls) apply_walls(nx, ny, nz, mask);
}

/* Random sequential addition of non-overlapping spheres of `radius` voxels.
 * Centres are uniform over x in [buffer + radius, nx - buffer - radius] and
 * periodic in y and z; a candidate is rejected if its centre lies closer than
 * 2*radius to an accepted centre (periodic in y, z).  Addition stops when the
 * voxel porosity of the packed slab x in [buffer, nx - buffer) reaches
 * `target_porosity` or after `max_failures` consecutive rejections (the RSA
 * jamming limit for spheres is a solid fraction near 0.38).  Voxel (x,y,z) is
 * solid when its centre lies inside a sphere.  Returns the number of spheres;
 * `porosity_out` gets the achieved slab porosity. */
long fm_synth_sphere_pack(int nx, int ny, int nz, double radius, double target_porosity,
                          int buffer, int walls, uint64_t seed, long max_failures,
                          uint8_t* mask, double* porosity_out)
{
    fm_rng r;
    rng_seed(&r, seed);
    const long n = (long)nx * ny * nz;
    memset(mask, 0, (size_t)n);
    const double lo = buffer + radius, hi = nx - buffer - radius - 1.0;
    if (hi <= lo || radius <= 0) { if (porosity_out) *porosity_out = 1.0; return 0; }
    /* hash grid over centres, cell size >= 2r */
    const double cs = 2.0 * radius;
    const int gx = (int)ceil(nx / cs) + 1, gy = (int)fmax(1.0, floor(ny / cs)), gz = (int)fmax(1.0, floor(nz / cs));
    const long ng = (long)gx * gy * gz;
    long* head = (long*)malloc(sizeof(long) * (size_t)ng);
    long cap = 1024, ns = 0;
    double* cen = (double*)malloc(sizeof(double) * 3 * (size_t)cap);
    long* next = (long*)malloc(sizeof(long) * (size_t)cap);
    if (!head || !cen || !next) { free(head); free(cen); free(next); return -1; }
    for (long i = 0; i < ng; ++i) head[i] = -1;

    const long slab = (long)(nx - 2 * buffer) * ny * nz;
    long solid = 0;
    const double r2 = radius * radius, d2min = cs * cs;
    const int ir = (int)ceil(radius);
    long fails = 0;
    while ((double)(slab - solid) / (double)slab > target_porosity && fails < max_failures) {
        const double cx = lo + (hi - lo) * rng_uniform(&r);
        const double cy = ny * rng_uniform(&r);
        const double cz = nz * rng_uniform(&r);
        const int hx = (int)(cx / cs), hy = (int)(cy / ny * gy) % gy, hz = (int)(cz / nz * gz) % gz;
        int ok = 1;
        for (int dz = -1; dz <= 1 && ok; ++dz)
            for (int dy = -1; dy <= 1 && ok; ++dy)
                for (int dx = -1; dx <= 1 && ok; ++dx) {
                    const int bx = hx + dx;
                    if (bx < 0 || bx >= gx) continue;
                    const int by = ((hy + dy) % gy + gy) % gy, bz = ((hz + dz) % gz + gz) % gz;
                    for (long s = head[bx + (long)gx * (by + (long)gy * bz)]; s >= 0; s = next[s]) {
                        double ex = cen[3 * s] - cx;
                        double ey = fabs(cen[3 * s + 1] - cy), ez = fabs(cen[3 * s + 2] - cz);
                        if (ey > 0.5 * ny) ey = ny - ey;
                        if (ez > 0.5 * nz) ez = nz - ez;
                        if (ex * ex + ey * ey + ez * ez < d2min) { ok = 0; break; }
                    }
                }
        if (!ok) { ++fails; continue; }
        fails = 0;
        if (ns == cap) {
            cap *= 2;
            double* c2 = (double*)realloc(cen, sizeof(double) * 3 * (size_t)cap);
            long* n2 = (long*)realloc(next, sizeof(long) * (size_t)cap);
            if (!c2 || !n2) { free(head); free(c2 ? c2 : cen); free(n2 ? n2 : next); return -1; }
            cen = c2; next = n2;
        }
        cen[3 * ns] = cx; cen[3 * ns + 1] = cy; cen[3 * ns + 2] = cz;
        const long b = hx + (long)gx * (hy + (long)gy * hz);
        next[ns] = head[b];
        head[b] = ns;
        ++ns;
        /* rasterise */
        for (int z = (int)floor(cz) - ir; z <= (int)ceil(cz) + ir; ++z)
            for (int y = (int)floor(cy) - ir; y <= (int)ceil(cy) + ir; ++y)
                for (int x = (int)floor(cx) - ir; x <= (int)ceil(cx) + ir; ++x) {
                    if (x < buffer || x >= nx - buffer) continue;
                    const double ddx = x - cx, ddy = y - cy, ddz = z - cz;
                    if (ddx * ddx + ddy * ddy + ddz * ddz > r2) continue;
                    const int yy = (y % ny + ny) % ny, zz = (z % nz + nz) % nz;
                    uint8_t* m = mask + x + (long)nx * (yy + (long)ny * zz);
                    if (!*m) { *m = 1; ++solid; }
                }
    }
    if (porosity_out) *porosity_out = (double)(slab - solid) / (double)slab;
    free(head); free(cen); free(next);
    if (walls) apply_walls(nx, ny, nz, mask);
    return ns;
}

/* Separable Gaussian smoothing (sigma in voxels, periodic, truncated at 4 sigma)
 * of i.i.d. uniform noise from `seed`; out[c] in float64.  Used for the
 * continuous solid-fraction field of the differentiation problem. */
int fm_synth_smooth_noise(int nx, int ny, int nz, double sigma, uint64_t seed, double* out)
{
    const long n = (long)nx * ny * nz;
    fm_synth_uniform(seed, n, out);
    const int R = (int)ceil(4.0 * sigma);
    double* k = (double*)malloc(sizeof(double) * (size_t)(2 * R + 1));
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    if (!k || !tmp) { free(k); free(tmp); return 1; }
    double ks = 0;
    for (int i = -R; i <= R; ++i) ks += (k[i + R] = exp(-0.5 * i * i / (sigma * sigma)));
    for (int i = 0; i <= 2 * R; ++i) k[i] /= ks;
    const int dims[3] = {nx, ny, nz};
    const long strides[3] = {1, nx, (long)nx * ny};
    for (int axis = 0; axis < 3; ++axis) {
        const int L = dims[axis];
        const long st = strides[axis];
        for (long c = 0; c < n; ++c) {
            const int pos = (int)((c / st) % L);
            double acc = 0;
            for (int i = -R; i <= R; ++i) {
                const int p = ((pos + i) % L + L) % L;
                acc += k[i + R] * out[c + (long)(p - pos) * st];
            }
            tmp[c] = acc;
        }
        memcpy(out, tmp, sizeof(double) * (size_t)n);
    }
    free(k); free(tmp);
    return 0;
}
