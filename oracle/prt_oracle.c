/*
 * CPU oracle for the diffuse path-tracing hot path — TEST INFRASTRUCTURE ONLY.
 * See prt_oracle.h for scope.  Only the test suite, the smoke check and the
 * benchmark's CPU-baseline leg load this code, always as the checker.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, pthreads).
 */
#include "prt_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <pthread.h>
#include <string.h>
#include <unistd.h>


/* ------------------------------------------------------------------------ */
/* Minimal parallel-for over pthreads (dynamic chunks of one index)          */
/* ------------------------------------------------------------------------ */

typedef void (*par_fn)(void* ctx, int index, int worker);

typedef struct {
    par_fn fn;
    void* ctx;
    int n;
    int next;
    int worker;
} par_job;

typedef struct {
    par_job* job;
    int worker;
} par_arg;

static void* par_main(void* p)
{
    par_arg* a = (par_arg*)p;
    for (;;)
    {
        int i = __atomic_fetch_add(&a->job->next, 1, __ATOMIC_RELAXED);
        if (i >= a->job->n) break;
        a->job->fn(a->job->ctx, i, a->worker);
    }
    return NULL;
}

static int worker_count(int nthreads)
{
    if (nthreads > 0) return nthreads;
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void par_for(int nthreads, int n, par_fn fn, void* ctx)
{
    int w = worker_count(nthreads);
    if (w > n) w = n;
    if (w <= 1)
    {
        for (int i = 0; i < n; ++i) fn(ctx, i, 0);
        return;
    }
    par_job job = {fn, ctx, n, 0, 0};
    pthread_t th[256];
    par_arg args[256];
    if (w > 256) w = 256;
    for (int k = 0; k < w; ++k) { args[k].job = &job; args[k].worker = k; }
    for (int k = 1; k < w; ++k) pthread_create(&th[k], NULL, par_main, &args[k]);
    par_main(&args[0]);
    for (int k = 1; k < w; ++k) pthread_join(th[k], NULL);
}

/* ------------------------------------------------------------------------ */
/* RNG: sampling/random_sampler.h:44-73, math/hash.h:23-72, math/math.h:179 */
/* ------------------------------------------------------------------------ */

static uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

/* murmurHash3Mix, math/hash.h:23-41 (shl/shr are logical, math/math.h:138-146) */
static uint32_t murmur_mix(uint32_t hash, uint32_t k)
{
    k *= 0xcc9e2d51u;
    k = rotl32(k, 15);
    k *= 0x1b873593u;
    hash ^= k;
    hash = rotl32(hash, 13) * 5u + 0xe6546b64u;
    return hash;
}

/* murmurHash3Finalize, math/hash.h:43-53 */
static uint32_t murmur_fin(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

/* RandomSampler::setSample with seed 0 (render/renderer.h:40-48) */
uint32_t or_rng_seed(int pass, int pixelIndex)
{
    uint32_t h = 0;
    h = murmur_mix(h, (uint32_t)pixelIndex);
    h = murmur_mix(h, (uint32_t)pass);
    return murmur_fin(h);
}

/* lcgNext, math/hash.h:65-72 */
uint32_t or_lcg_next(uint32_t s) { return s * 1664525u + 1013904223u; }

/* toFloatUnorm, math/math.h:179: uint32 -> float rounds to nearest, then 2^-32 */
float or_unorm(uint32_t s) { return (float)s * 0x1.0p-32f; }

static void get2d(uint32_t* st, double* x, double* y)
{
    *st = or_lcg_next(*st);
    *x = (double)or_unorm(*st);
    *st = or_lcg_next(*st);
    *y = (double)or_unorm(*st);
}

/* ------------------------------------------------------------------------ */
/* Camera (float arithmetic, as the reference computes it on the host)      */
/* ------------------------------------------------------------------------ */

typedef struct { float x, y, z; } f3;

static f3 f3m(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static f3 f3add(f3 a, f3 b) { return f3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static f3 f3scale(f3 a, float s) { return f3m(a.x * s, a.y * s, a.z * s); }
static float f3dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static f3 f3cross(f3 a, f3 b) { return f3m(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

/* rotate(vec, axis, angle), math/vec3.h:409-412 */
static f3 f3rotate(f3 vec, f3 axis, float angle)
{
    float c = cosf(angle), s = sinf(angle);
    f3 a = f3scale(vec, c);
    f3 b = f3scale(f3scale(axis, f3dot(axis, vec)), 1.0f - c);
    f3 d = f3scale(f3cross(vec, axis), s);
    return f3add(f3add(a, b), d);
}

/* basis * (a.x, a.y, a.z) = a.x U + a.y V + a.z N, math/basis3.h:120-124 */
static f3 basis_mul(f3 U, f3 V, f3 N, float ax, float ay, float az)
{
    return f3add(f3add(f3scale(U, ax), f3scale(V, ay)), f3scale(N, az));
}

static void store3(float* d, f3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }

/* RenderWindow::makeCamera (main/render/render_window.cpp:307-325) with
 * Basis3f(one).rotateV(angleY).rotateU(angleX) (math/basis3.h:63-79), then
 * PinholeCamera / ThinLensCamera construction (camera/pinhole_camera.h:34-47,
 * camera/thin_lens_camera.h:29-36); the pinhole camera is selected when the
 * lens radius is 0 (render/device_cpu_impl.cpp:86-97). */
void or_camera_from_view(const or_view* v, float aspect, or_camera* cam)
{
    f3 V = f3m(0, 1, 0), N = f3m(0, 0, 1);   /* Basis3f(one); U = (1,0,0) is replaced below */
    /* rotateV(angleY): N' = rotate(N, V, a); U' = cross(V, N') */
    f3 N1 = f3rotate(N, V, v->angleY);
    f3 U1 = f3cross(V, N1);
    f3 V1 = V;
    /* rotateU(angleX): V'' = rotate(V', U', b); N'' = cross(U', V'') */
    f3 V2 = f3rotate(V1, U1, v->angleX);
    f3 N2 = f3cross(U1, V2);
    f3 U2 = U1;

    float hh = tanf(0.5f * v->fovY);
    float hw = hh * aspect;
    store3(cam->origin, f3m(v->pos[0], v->pos[1], v->pos[2]));
    store3(cam->U, U2);
    store3(cam->V, V2);
    store3(cam->N, N2);
    store3(cam->imageO, basis_mul(U2, V2, N2, -hw, hh, -1.0f));
    store3(cam->imageDx, basis_mul(U2, V2, N2, 2.0f * hw, 0.0f, 0.0f));
    store3(cam->imageDy, basis_mul(U2, V2, N2, 0.0f, (float)(-2.0 * (double)hh), 0.0f));
    cam->lensRadius = v->radius;
    cam->focalDistance = v->focus;
    cam->thinLens = v->radius != 0.0f;
}

/* ------------------------------------------------------------------------ */
/* FP64 vector helpers                                                       */
/* ------------------------------------------------------------------------ */

static void d3sub(const double* a, const double* b, double* r) { r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2]; }
static double d3dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void d3cross(const double* a, const double* b, double* r)
{
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    r[0] = x; r[1] = y; r[2] = z;
}
static void d3normalize(double* a)
{
    double l = sqrt(d3dot(a, a));
    if (l > 0) { a[0] /= l; a[1] /= l; a[2] /= l; }
}

/* ------------------------------------------------------------------------ */
/* Scene + FP64 BVH                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    double lo[3], hi[3];
    int first;   /* leaf: first index into order[]; internal: left child */
    int count;   /* leaf: triangle count (>0); internal: 0 */
} bnode;

struct or_scene {
    int nt, nv;
    double* v;      /* nv*3 */
    int* idx;       /* nt*3 */
    bnode* nodes;
    int nnodes;
    int* order;     /* nt */
    double* cent;   /* nt*3 */
    double* tlo;    /* nt*3 triangle boxes */
    double* thi;
};

static void tri_verts(const or_scene* s, int p, const double** a, const double** b, const double** c)
{
    *a = s->v + 3 * s->idx[3 * p + 0];
    *b = s->v + 3 * s->idx[3 * p + 1];
    *c = s->v + 3 * s->idx[3 * p + 2];
}

static int cmp_axis;
static const double* cmp_cent;

static int cmp_tri(const void* A, const void* B)
{
    int a = *(const int*)A, b = *(const int*)B;
    double ca = cmp_cent[3 * a + cmp_axis], cb = cmp_cent[3 * b + cmp_axis];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
    return (a > b) - (a < b);
}

static int build_node(or_scene* s, int first, int count, int* next)
{
    int ni = (*next)++;
    bnode* n = &s->nodes[ni];
    int k;
    for (k = 0; k < 3; ++k) { n->lo[k] = DBL_MAX; n->hi[k] = -DBL_MAX; }
    double clo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, chi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int i = first; i < first + count; ++i)
    {
        int p = s->order[i];
        for (k = 0; k < 3; ++k)
        {
            if (s->tlo[3 * p + k] < n->lo[k]) n->lo[k] = s->tlo[3 * p + k];
            if (s->thi[3 * p + k] > n->hi[k]) n->hi[k] = s->thi[3 * p + k];
            double c = s->cent[3 * p + k];
            if (c < clo[k]) clo[k] = c;
            if (c > chi[k]) chi[k] = c;
        }
    }
    if (count <= 4)
    {
        n->first = first;
        n->count = count;
        return ni;
    }
    int axis = 0;
    for (k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
    cmp_axis = axis;
    cmp_cent = s->cent;
    qsort(s->order + first, (size_t)count, sizeof(int), cmp_tri);
    int half = count / 2;
    n->count = 0;
    int l = build_node(s, first, half, next);
    int r = build_node(s, first + half, count - half, next);
    (void)r;
    s->nodes[ni].first = l;   /* children are l and r; r == l + size(l) */
    s->nodes[ni].count = -r;  /* store right child as negative to keep the struct small */
    return ni;
}

or_scene* or_scene_create(const float* positions, int nv, const int* indices, int nt)
{
    if (nt < 0 || nv < 0 || (nt > 0 && (!positions || !indices))) return NULL;
    for (int i = 0; i < 3 * nt; ++i)
        if (indices[i] < 0 || indices[i] >= nv) return NULL;
    or_scene* s = (or_scene*)calloc(1, sizeof(or_scene));
    s->nt = nt;
    s->nv = nv;
    s->v = (double*)malloc(sizeof(double) * 3 * (size_t)(nv > 0 ? nv : 1));
    for (int i = 0; i < 3 * nv; ++i) s->v[i] = positions[i];
    s->idx = (int*)malloc(sizeof(int) * 3 * (size_t)(nt > 0 ? nt : 1));
    if (nt) memcpy(s->idx, indices, sizeof(int) * 3 * (size_t)nt);
    s->order = (int*)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    s->cent = (double*)malloc(sizeof(double) * 3 * (size_t)(nt > 0 ? nt : 1));
    s->tlo = (double*)malloc(sizeof(double) * 3 * (size_t)(nt > 0 ? nt : 1));
    s->thi = (double*)malloc(sizeof(double) * 3 * (size_t)(nt > 0 ? nt : 1));
    for (int p = 0; p < nt; ++p)
    {
        const double *a, *b, *c;
        tri_verts(s, p, &a, &b, &c);
        for (int k = 0; k < 3; ++k)
        {
            double lo = fmin(a[k], fmin(b[k], c[k])), hi = fmax(a[k], fmax(b[k], c[k]));
            double pad = 1e-9 * (fabs(lo) + fabs(hi)) + 1e-300;
            s->tlo[3 * p + k] = lo - pad;
            s->thi[3 * p + k] = hi + pad;
            s->cent[3 * p + k] = 0.5 * (lo + hi);
        }
        s->order[p] = p;
    }
    s->nodes = (bnode*)malloc(sizeof(bnode) * (size_t)(2 * (nt > 0 ? nt : 1)));
    int next = 0;
    if (nt > 0) build_node(s, 0, nt, &next);
    s->nnodes = next;
    return s;
}

void or_scene_destroy(or_scene* s)
{
    if (!s) return;
    free(s->v); free(s->idx); free(s->order); free(s->cent); free(s->tlo); free(s->thi); free(s->nodes);
    free(s);
}

int or_scene_tri_count(const or_scene* s) { return s ? s->nt : 0; }

/* Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013) in FP64.
 * Barycentrics follow the reference CPU convention: u weights v1, v weights v2
 * (geometry/triangle_mesh.cpp:69-71). */
typedef struct {
    double org[3];
    int kx, ky, kz;
    double Sx, Sy, Sz;
} wt_ray;

static void wt_setup(wt_ray* r, const double org[3], const double dir[3])
{
    int kz = 0;
    if (fabs(dir[1]) > fabs(dir[kz])) kz = 1;
    if (fabs(dir[2]) > fabs(dir[kz])) kz = 2;
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (dir[kz] < 0) { int t = kx; kx = ky; ky = t; }
    r->kx = kx; r->ky = ky; r->kz = kz;
    r->Sx = dir[kx] / dir[kz];
    r->Sy = dir[ky] / dir[kz];
    r->Sz = 1.0 / dir[kz];
    memcpy(r->org, org, sizeof(double) * 3);
}

/* returns 1 with t,b1,b2 and the smallest barycentric when hit in (tnear, tfar] */
static int wt_hit(const wt_ray* r, const double* v0, const double* v1, const double* v2,
                  double tnear, double tfar, double* t, double* b1, double* b2, double* bmin)
{
    double A[3], B[3], C[3];
    d3sub(v0, r->org, A);
    d3sub(v1, r->org, B);
    d3sub(v2, r->org, C);
    double Ax = A[r->kx] - r->Sx * A[r->kz], Ay = A[r->ky] - r->Sy * A[r->kz];
    double Bx = B[r->kx] - r->Sx * B[r->kz], By = B[r->ky] - r->Sy * B[r->kz];
    double Cx = C[r->kx] - r->Sx * C[r->kz], Cy = C[r->ky] - r->Sy * C[r->kz];
    double U = Cx * By - Cy * Bx;
    double V = Ax * Cy - Ay * Cx;
    double W = Bx * Ay - By * Ax;
    if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return 0;
    double det = U + V + W;
    if (det == 0) return 0;
    double Az = r->Sz * A[r->kz], Bz = r->Sz * B[r->kz], Cz = r->Sz * C[r->kz];
    double T = U * Az + V * Bz + W * Cz;
    double tt = T / det;
    if (!(tt > tnear) || !(tt <= tfar)) return 0;
    *t = tt;
    *b1 = V / det;
    *b2 = W / det;
    double b0 = U / det;
    double m = b0 < *b1 ? b0 : *b1;
    *bmin = m < *b2 ? m : *b2;
    return 1;
}

static int box_hit(const bnode* n, const double org[3], const double inv[3], double tnear, double tfar)
{
    double t0 = tnear, t1 = tfar;
    for (int k = 0; k < 3; ++k)
    {
        double a = (n->lo[k] - org[k]) * inv[k];
        double b = (n->hi[k] - org[k]) * inv[k];
        if (a != a) a = -DBL_MAX;   /* 0 * inf inside the slab */
        if (b != b) b = DBL_MAX;
        double lo = a < b ? a : b, hi = a < b ? b : a;
        if (lo > t0) t0 = lo;
        if (hi < t1) t1 = hi;
    }
    return t0 <= t1 * (1.0 + 1e-12) + 1e-300;
}

/* mode 0: closest hit; mode 1: any hit; mode 2: any hit other than `exclude`
 * within (tnear, tfar] (used for the near-tie check) */
static int traverse(const or_scene* s, const double org[3], const double dir[3], double tnear, double tfar,
                    int mode, int exclude, or_hit* out)
{
    if (s->nt == 0) return 0;
    wt_ray wr;
    wt_setup(&wr, org, dir);
    double inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0 / dir[k];
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    int found = 0;
    double best = tfar, bu = 0, bv = 0, bmin = 1;
    int bprim = -1;
    while (sp > 0)
    {
        const bnode* n = &s->nodes[stack[--sp]];
        if (!box_hit(n, org, inv, tnear, best)) continue;
        if (n->count > 0)
        {
            for (int i = n->first; i < n->first + n->count; ++i)
            {
                int p = s->order[i];
                if (mode == 2 && p == exclude) continue;
                const double *a, *b, *c;
                tri_verts(s, p, &a, &b, &c);
                double t, u, v, m;
                if (!wt_hit(&wr, a, b, c, tnear, best, &t, &u, &v, &m)) continue;
                if (mode != 0) { if (out) { out->t = t; out->primId = p; } return 1; }
                /* exact ties resolve to the lower primitive id (order independent) */
                if (found && t == best && p > bprim) continue;
                found = 1; best = t; bu = u; bv = v; bprim = p; bmin = m;
            }
        }
        else
        {
            int l = n->first, r = -n->count;
            /* visit the nearer child first: push the farther one first */
            double dl = (s->nodes[l].lo[0] + s->nodes[l].hi[0]) * dir[0] + (s->nodes[l].lo[1] + s->nodes[l].hi[1]) * dir[1] + (s->nodes[l].lo[2] + s->nodes[l].hi[2]) * dir[2];
            double dr = (s->nodes[r].lo[0] + s->nodes[r].hi[0]) * dir[0] + (s->nodes[r].lo[1] + s->nodes[r].hi[1]) * dir[1] + (s->nodes[r].lo[2] + s->nodes[r].hi[2]) * dir[2];
            if (sp + 2 > 128) return -1;
            if (dl < dr) { stack[sp++] = r; stack[sp++] = l; }
            else { stack[sp++] = l; stack[sp++] = r; }
        }
    }
    if (found && out)
    {
        out->t = best; out->primId = bprim; out->u = bu; out->v = bv;
        out->grazing = bmin < 1e-5;
    }
    return found;
}

int or_intersect(const or_scene* s, const double org[3], const double dir[3], double tnear, double tfar, or_hit* hit)
{
    or_hit h;
    memset(&h, 0, sizeof(h));
    int r = traverse(s, org, dir, tnear, tfar, 0, -1, &h);
    if (r > 0 && hit) *hit = h;
    return r > 0;
}

int or_occluded(const or_scene* s, const double org[3], const double dir[3], double tnear, double tfar)
{
    return traverse(s, org, dir, tnear, tfar, 1, -1, NULL) > 0;
}

typedef struct {
    const or_scene* s;
    const float* rays;
    float* hits;
    int* flags;
    int n;
} isect_ctx;

static void isect_one(void* vctx, int chunk, int worker)
{
    (void)worker;
    isect_ctx* c = (isect_ctx*)vctx;
    int i0 = chunk * 256, i1 = i0 + 256 < c->n ? i0 + 256 : c->n;
    for (int i = i0; i < i1; ++i)
    {
        const float* r = c->rays + 8 * (size_t)i;
        double org[3] = {r[0], r[1], r[2]}, dir[3] = {r[4], r[5], r[6]};
        double tnear = r[3], tfar = r[7];
        or_hit h;
        int ok = or_intersect(c->s, org, dir, tnear, tfar, &h);
        float* o = c->hits + 4 * (size_t)i;
        if (ok)
        {
            int prim = h.primId;
            o[0] = (float)h.t;
            memcpy(&o[1], &prim, 4);
            o[2] = (float)h.u;
            o[3] = (float)h.v;
        }
        else
        {
            int neg = -1;
            o[0] = -1.0f;
            memcpy(&o[1], &neg, 4);
            o[2] = 0;
            o[3] = 0;
        }
        if (c->flags)
        {
            int g = ok ? h.grazing : 0;
            if (ok && !g)
            {
                /* near-tie: another triangle within a relative 1e-6 of t */
                double band = h.t * (1.0 + 1e-6) + 1e-12;
                or_hit h2;
                if (traverse(c->s, org, dir, tnear, band, 2, h.primId, &h2) > 0) g = 1;
            }
            if (!ok)
            {
                /* a miss is grazing when a direction perturbed by 1e-6 (relative)
                 * along any axis hits something */
                for (int k = 0; k < 3 && !g; ++k)
                    for (int sgn = -1; sgn <= 1 && !g; sgn += 2)
                    {
                        double d2[3] = {dir[0], dir[1], dir[2]};
                        d2[k] += sgn * 1e-6 * (fabs(dir[0]) + fabs(dir[1]) + fabs(dir[2]));
                        if (or_occluded(c->s, org, d2, tnear, tfar)) g = 1;
                    }
            }
            c->flags[i] = g;
        }
    }
}

void or_intersect_rays(const or_scene* s, const float* rays, int n, float* hits, int* flags, int nthreads)
{
    isect_ctx c = {s, rays, hits, flags, n};
    par_for(nthreads, (n + 255) / 256, isect_one, &c);
}

typedef struct {
    const or_scene* s;
    const float* rays;
    float* out;
    int n;
} occl_ctx;

static void occl_one(void* vctx, int chunk, int worker)
{
    (void)worker;
    occl_ctx* c = (occl_ctx*)vctx;
    int i0 = chunk * 256, i1 = i0 + 256 < c->n ? i0 + 256 : c->n;
    for (int i = i0; i < i1; ++i)
    {
        const float* r = c->rays + 8 * (size_t)i;
        double org[3] = {r[0], r[1], r[2]}, dir[3] = {r[4], r[5], r[6]};
        or_hit h;
        int ok = traverse(c->s, org, dir, r[3], r[7], 1, -1, &h) > 0;
        c->out[i] = ok ? (float)h.t : -1.0f;
    }
}

void or_occluded_rays(const or_scene* s, const float* rays, int n, float* out, int nthreads)
{
    occl_ctx c = {s, rays, out, n};
    par_for(nthreads, (n + 255) / 256, occl_one, &c);
}

/* ------------------------------------------------------------------------ */
/* Sampling: sampling/shape_sampler.h:50-74 (cosine), :114-124 (disk)        */
/* ------------------------------------------------------------------------ */

void or_cosine_sample_hemisphere(double sx, double sy, double out[3])
{
    double cosTheta = sqrt(sx);
    double sinTheta = sqrt(1.0 - sx);
    double phi = 2.0 * M_PI * sy;
    out[0] = cos(phi) * sinTheta;
    out[1] = sin(phi) * sinTheta;
    out[2] = cosTheta;
}

static void uniform_sample_disk(double sx, double sy, double* x, double* y)
{
    double r = sqrt(sx);
    double th = 2.0 * M_PI * sy;
    *x = r * cos(th);
    *y = r * sin(th);
}

/* makeFrame, math/basis3.h:128-137 */
void or_make_frame(const double N[3], double U[3], double V[3])
{
    double U0[3] = {0.0, N[2], -N[1]};
    double U1[3] = {-N[2], 0.0, N[0]};
    if (d3dot(U0, U0) > d3dot(U1, U1)) memcpy(U, U0, sizeof(U0));
    else memcpy(U, U1, sizeof(U1));
    d3normalize(U);
    d3cross(N, U, V);
    d3normalize(V);
}

/* TriangleMesh::postIntersect without normals/uvs (geometry/triangle_mesh.cpp:59-100)
 * and Ray::getHitPoint(eps) (core/ray.h:71-76). */
void or_post_intersect(const or_scene* s, const double org[3], const double dir[3], double t, int primId,
                       double p[3], double* eps, double Ng[3])
{
    for (int k = 0; k < 3; ++k) p[k] = org[k] + t * dir[k];
    double m = fabs(p[0]);
    if (fabs(p[1]) > m) m = fabs(p[1]);
    if (fabs(p[2]) > m) m = fabs(p[2]);
    *eps = (t > m ? t : m) * 0x1.fp-18;
    const double *a, *b, *c;
    tri_verts(s, primId, &a, &b, &c);
    double e1[3], e2[3];
    d3sub(b, a, e1);
    d3sub(c, a, e2);
    d3cross(e1, e2, Ng);
    d3normalize(Ng);
    if (d3dot(Ng, dir) > 0) { Ng[0] = -Ng[0]; Ng[1] = -Ng[1]; Ng[2] = -Ng[2]; }
}

/* ------------------------------------------------------------------------ */
/* Path re-evaluation: render/renderer_single.h:107-131 +                    */
/* render/diffuse_integrator_single.h:41-69                                   */
/* ------------------------------------------------------------------------ */

static void camera_ray(const or_camera* cam, double ix, double iy, double lx, double ly, double org[3], double dir[3])
{
    double d[3];
    if (!cam->thinLens)
    {
        /* camera/pinhole_camera.h:50-54 */
        for (int k = 0; k < 3; ++k)
        {
            d[k] = (double)cam->imageO[k] + ix * cam->imageDx[k] + iy * cam->imageDy[k];
            org[k] = cam->origin[k];
        }
    }
    else
    {
        /* camera/thin_lens_camera.h:38-44 */
        double dx, dy;
        uniform_sample_disk(lx, ly, &dx, &dy);
        dx *= cam->lensRadius;
        dy *= cam->lensRadius;
        for (int k = 0; k < 3; ++k)
        {
            double begin = (double)cam->origin[k] + dx * cam->U[k] + dy * cam->V[k];
            double end = (double)cam->origin[k] + (double)cam->focalDistance *
                         ((double)cam->imageO[k] + ix * cam->imageDx[k] + iy * cam->imageDy[k]);
            org[k] = begin;
            d[k] = end - begin;
        }
    }
    d3normalize(d);
    memcpy(dir, d, sizeof(d));
}

/* Evaluates one path; returns its radiance.  prims (nullable, maxDepth
 * entries) receives the primitive ids whose albedo scaled the throughput. */
static double eval_path(const or_scene* s, const or_camera* cam, int W, int H, int x, int y, int pass,
                        int maxDepth, const float* albedo, double sky, int64_t* rays, int* prims, int* nprims,
                        double* through)
{
    int pixel = x + y * W;
    uint32_t st = or_rng_seed(pass, pixel);
    double jx, jy, lx, ly;
    get2d(&st, &jx, &jy);   /* sampleDimPixel */
    get2d(&st, &lx, &ly);   /* sampleDimLens */
    double ix = ((double)x + jx) / (double)W;
    double iy = ((double)y + jy) / (double)H;
    double org[3], dir[3];
    camera_ray(cam, ix, iy, lx, ly, org, dir);

    double Lw = 1.0;
    int depth = 0, hit = 0, np = 0;
    for (;;)
    {
        or_hit h;
        hit = or_intersect(s, org, dir, 0.0, DBL_MAX, &h);
        (*rays)++;
        if (!hit || depth == maxDepth) break;
        double a = albedo ? (double)albedo[h.primId] : (double)0.8f;
        Lw *= a;
        if (prims) prims[np] = h.primId;
        np++;
        double p[3], eps, Ng[3], U[3], V[3], l[3], sx, sy;
        or_post_intersect(s, org, dir, h.t, h.primId, p, &eps, Ng);
        or_make_frame(Ng, U, V);
        get2d(&st, &sx, &sy);
        or_cosine_sample_hemisphere(sx, sy, l);
        for (int k = 0; k < 3; ++k)
        {
            double nd = l[0] * U[k] + l[1] * V[k] + l[2] * Ng[k];
            dir[k] = nd;
        }
        /* Ray::init(org, dir, near) offsets the origin (core/ray.h:47-52) */
        for (int k = 0; k < 3; ++k) org[k] = p[k] + eps * dir[k];
        depth++;
    }
    if (nprims) *nprims = np;
    if (through) *through = Lw;
    return hit ? 0.0 : Lw * sky;
}

void or_primary_rays(const or_camera* cam, int W, int H, int pass, float* rays)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            int pixel = x + y * W;
            uint32_t st = or_rng_seed(pass, pixel);
            double jx, jy, lx, ly;
            get2d(&st, &jx, &jy);
            get2d(&st, &lx, &ly);
            double org[3], dir[3];
            camera_ray(cam, ((double)x + jx) / W, ((double)y + jy) / H, lx, ly, org, dir);
            float* r = rays + 8 * (size_t)pixel;
            r[0] = (float)org[0]; r[1] = (float)org[1]; r[2] = (float)org[2]; r[3] = 0.0f;
            r[4] = (float)dir[0]; r[5] = (float)dir[1]; r[6] = (float)dir[2]; r[7] = FLT_MAX;
        }
}

/* Diffuse path with next-event estimation toward the sky
 * (render/diffuse2_integrator_single.h:41-90): at every hit before maxDepth a
 * cosine-distributed shadow ray is tested for any occluder and, if it
 * escapes, adds throughput * 0.5; the extension ray adds throughput * 0.5 on
 * escape after the first bounce and throughput * 1 from the camera (fixed MIS
 * weights).  Four sample dimensions per bounce: shadow (2), extension (2).
 * Shadow rays count as rays, as occluded() does in the reference. */
static double eval_path_nee(const or_scene* s, const or_camera* cam, int W, int H, int x, int y, int pass,
                            int maxDepth, const float* albedo, double sky, int64_t* rays)
{
    int pixel = x + y * W;
    uint32_t st = or_rng_seed(pass, pixel);
    double jx, jy, lx, ly;
    get2d(&st, &jx, &jy);
    get2d(&st, &lx, &ly);
    double org[3], dir[3];
    camera_ray(cam, ((double)x + jx) / (double)W, ((double)y + jy) / (double)H, lx, ly, org, dir);
    double L = 0.0, thr = 1.0;
    for (int depth = 0;; ++depth)
    {
        or_hit h;
        int hit = or_intersect(s, org, dir, 0.0, DBL_MAX, &h);
        (*rays)++;
        if (!hit)
        {
            L += thr * sky * (depth > 0 ? 0.5 : 1.0);
            break;
        }
        if (depth == maxDepth) break;
        double p[3], eps, Ng[3], U[3], V[3], l[3], sx, sy;
        or_post_intersect(s, org, dir, h.t, h.primId, p, &eps, Ng);
        or_make_frame(Ng, U, V);
        thr *= albedo ? (double)albedo[h.primId] : (double)0.8f;
        /* shadow ray */
        get2d(&st, &sx, &sy);
        or_cosine_sample_hemisphere(sx, sy, l);
        double so[3], sd[3];
        for (int k = 0; k < 3; ++k) sd[k] = l[0] * U[k] + l[1] * V[k] + l[2] * Ng[k];
        for (int k = 0; k < 3; ++k) so[k] = p[k] + eps * sd[k];
        (*rays)++;
        if (!or_occluded(s, so, sd, 0.0, DBL_MAX)) L += thr * sky * 0.5;
        /* extension ray */
        get2d(&st, &sx, &sy);
        or_cosine_sample_hemisphere(sx, sy, l);
        for (int k = 0; k < 3; ++k) dir[k] = l[0] * U[k] + l[1] * V[k] + l[2] * Ng[k];
        for (int k = 0; k < 3; ++k) org[k] = p[k] + eps * dir[k];
    }
    return L;
}

typedef struct {
    const or_scene* s;
    const or_camera* cam;
    int W, H, pass0, npass, maxDepth;
    const float* albedo;
    double sky;
    double* accum;
    int nee;
    int64_t rows_rays[1];
    int64_t* rays;          /* per row */
    const double* dL;       /* backward only */
    double* part;           /* backward: per worker (ntri + 1) doubles */
    int** prims;            /* backward: per worker scratch */
} render_ctx;

static void render_row(void* vctx, int y, int worker)
{
    (void)worker;
    render_ctx* c = (render_ctx*)vctx;
    int64_t rays = 0;
    for (int x = 0; x < c->W; ++x)
    {
        double* a = c->accum + 4 * ((size_t)y * c->W + x);
        for (int p = 0; p < c->npass; ++p)
        {
            double v = c->nee ? eval_path_nee(c->s, c->cam, c->W, c->H, x, y, c->pass0 + p, c->maxDepth, c->albedo,
                                              c->sky, &rays)
                              : eval_path(c->s, c->cam, c->W, c->H, x, y, c->pass0 + p, c->maxDepth, c->albedo,
                                          c->sky, &rays, NULL, NULL, NULL);
            a[0] += v; a[1] += v; a[2] += v; a[3] += 1.0;
        }
    }
    c->rays[y] = rays;
}

int64_t or_render(const or_scene* s, const or_camera* cam, int W, int H, int pass0, int npass, int maxDepth,
                  const float* albedo, float sky, double* accum, int nthreads)
{
    return or_render_ex(s, cam, W, H, pass0, npass, maxDepth, albedo, sky, accum, nthreads, 0);
}

int64_t or_render_ex(const or_scene* s, const or_camera* cam, int W, int H, int pass0, int npass, int maxDepth,
                     const float* albedo, float sky, double* accum, int nthreads, int nee)
{
    render_ctx c;
    memset(&c, 0, sizeof(c));
    c.s = s; c.cam = cam; c.W = W; c.H = H; c.pass0 = pass0; c.npass = npass; c.maxDepth = maxDepth;
    c.albedo = albedo; c.sky = sky; c.accum = accum; c.nee = nee;
    c.rays = (int64_t*)calloc((size_t)(H > 0 ? H : 1), sizeof(int64_t));
    par_for(nthreads, H, render_row, &c);
    int64_t total = 0;
    for (int y = 0; y < H; ++y) total += c.rays[y];
    free(c.rays);
    return total;
}

typedef struct {
    const or_scene* s;
    const or_camera* cam;
    int W, H, pass0, npass, maxDepth, nee;
    const float* albedo;
    double sky;
    const int* pixels;
    double* out;
    int64_t* rays;
} pixels_ctx;

/* One listed pixel, its passes in order: the same per-pixel sums as
 * render_row (RendererSingle::renderTile, render/renderer_single.h:107-131). */
static void render_listed_pixel(void* vctx, int i, int worker)
{
    (void)worker;
    pixels_ctx* c = (pixels_ctx*)vctx;
    int pixel = c->pixels[i];
    int x = pixel % c->W, y = pixel / c->W;
    int64_t rays = 0;
    double* a = c->out + 4 * (size_t)i;
    a[0] = a[1] = a[2] = a[3] = 0.0;
    for (int p = 0; p < c->npass; ++p)
    {
        double v = c->nee ? eval_path_nee(c->s, c->cam, c->W, c->H, x, y, c->pass0 + p, c->maxDepth, c->albedo,
                                          c->sky, &rays)
                          : eval_path(c->s, c->cam, c->W, c->H, x, y, c->pass0 + p, c->maxDepth, c->albedo,
                                      c->sky, &rays, NULL, NULL, NULL);
        a[0] += v; a[1] += v; a[2] += v; a[3] += 1.0;
    }
    c->rays[i] = rays;
}

int64_t or_render_pixels(const or_scene* s, const or_camera* cam, int W, int H, const int* pixels, int n,
                         int pass0, int npass, int maxDepth, const float* albedo, float sky, double* out,
                         int64_t* rays_out, int nthreads, int nee)
{
    if (n <= 0) return 0;
    for (int i = 0; i < n; ++i)
        if (pixels[i] < 0 || (int64_t)pixels[i] >= (int64_t)W * H) return -1;
    pixels_ctx c;
    memset(&c, 0, sizeof(c));
    c.s = s; c.cam = cam; c.W = W; c.H = H; c.pass0 = pass0; c.npass = npass; c.maxDepth = maxDepth;
    c.nee = nee; c.albedo = albedo; c.sky = sky; c.pixels = pixels; c.out = out;
    c.rays = rays_out ? rays_out : (int64_t*)calloc((size_t)n, sizeof(int64_t));
    par_for(nthreads, n, render_listed_pixel, &c);
    int64_t total = 0;
    for (int i = 0; i < n; ++i) total += c.rays[i];
    if (!rays_out) free(c.rays);
    return total;
}

static void backward_row(void* vctx, int y, int worker)
{
    render_ctx* c = (render_ctx*)vctx;
    int ntri = c->s->nt;
    double* g_alb = c->part + (size_t)worker * (size_t)(ntri + 1);
    int* prims = c->prims[worker];
    int64_t rays = 0;
    for (int x = 0; x < c->W; ++x)
    {
        const double* gp = c->dL + 3 * ((size_t)y * c->W + x);
        double g = gp[0] + gp[1] + gp[2];
        if (g == 0.0) continue;
        for (int p = 0; p < c->npass; ++p)
        {
            int np = 0;
            double Lw = 0;
            double v = eval_path(c->s, c->cam, c->W, c->H, x, y, c->pass0 + p, c->maxDepth, c->albedo, c->sky,
                                 &rays, prims, &np, &Lw);
            if (v == 0.0) continue;
            g_alb[ntri] += g * Lw;   /* d radiance / d sky = product of albedos */
            for (int k = 0; k < np; ++k)
            {
                double a = c->albedo ? (double)c->albedo[prims[k]] : (double)0.8f;
                g_alb[prims[k]] += g * v / a;
            }
        }
    }
}

void or_render_backward(const or_scene* s, const or_camera* cam, int W, int H, int pass0, int npass, int maxDepth,
                        const float* albedo, float sky, const double* dL_dsum, double* d_albedo, double* d_sky,
                        int nthreads)
{
    int nw = worker_count(nthreads);
    if (nw > 256) nw = 256;
    if (nw > H) nw = H > 0 ? H : 1;
    int ntri = s->nt;
    render_ctx c;
    memset(&c, 0, sizeof(c));
    c.s = s; c.cam = cam; c.W = W; c.H = H; c.pass0 = pass0; c.npass = npass; c.maxDepth = maxDepth;
    c.albedo = albedo; c.sky = sky; c.dL = dL_dsum;
    c.part = (double*)calloc((size_t)nw * (size_t)(ntri + 1), sizeof(double));
    c.prims = (int**)malloc(sizeof(int*) * (size_t)nw);
    for (int k = 0; k < nw; ++k) c.prims[k] = (int*)malloc(sizeof(int) * (size_t)(maxDepth + 1));
    par_for(nw, H, backward_row, &c);
    for (int i = 0; i <= ntri; ++i)
    {
        double acc = 0;
        for (int t = 0; t < nw; ++t) acc += c.part[(size_t)t * (ntri + 1) + i];
        if (i < ntri) d_albedo[i] = acc;
        else *d_sky = acc;
    }
    for (int k = 0; k < nw; ++k) free(c.prims[k]);
    free(c.prims);
    free(c.part);
}
