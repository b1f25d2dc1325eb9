/*
 * yr_oracle.c — TEST ORACLE: plain-C restatement of the reference's traversal,
 * sampler, camera and film arithmetic (QiuRuhai/YaoRay). It is used by the
 * tests to check the CUDA kernels and by the benchmark's CPU-baseline leg; it
 * is pinned against the compiled reference (oracle/_ref) and the golden
 * vectors in tests/golden. Compile with -ffp-contract=off and no -march so
 * that every float operation rounds like the reference's SSE2 build.
 */
#include "yr_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------- vector math */

/* Dot: (ax*bx + ay*by) + az*bz (include/yaoray/core/vec.hpp:155-157). */
static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Cross (vec.hpp:159-165). */
static void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

static const float* vpos(const yo_geometry* g, uint64_t i) {
    return (const float*)((const char*)g->positions + (int64_t)i * g->vertex_stride);
}

/* PrecomputeRayBounds (include/yaoray/core/bounds.hpp:56-66). */
typedef struct ray_pre {
    float o[3], d[3], inv[3];
    int neg[3];
} ray_pre;

static void precompute(ray_pre* r, const float* o, const float* d) {
    for (int a = 0; a < 3; ++a) {
        r->o[a] = o[a];
        r->d[a] = d[a];
        r->inv[a] = 1.0f / d[a];
        r->neg[a] = signbit(r->inv[a]) ? 1 : 0;
    }
}

/* IntersectBounds (bounds.hpp:68-90). */
static int intersect_bounds(const yo_node* n, const ray_pre* r, float t_min, float t_max, float* entry) {
    for (int a = 0; a < 3; ++a) {
        const float nb = r->neg[a] ? n->hi[a] : n->lo[a];
        const float fb = r->neg[a] ? n->lo[a] : n->hi[a];
        const float an = (nb - r->o[a]) * r->inv[a];
        const float af = (fb - r->o[a]) * r->inv[a];
        t_min = an > t_min ? an : t_min;
        t_max = af < t_max ? af : t_max;
    }
    *entry = t_min;
    return t_max >= t_min;
}

static yo_hit miss_hit(float t_max) {
    yo_hit h;
    h.hit = 0;
    h.t = t_max;
    h.triangle_index = -1;
    h.mesh_primitive = -1;
    h.instance = -1;
    h.sphere = -1;
    h.u = 0.0f;
    h.v = 0.0f;
    return h;
}

/* IntersectTriangle (src/accel/bvh_traversal.cpp:52-121). */
static void intersect_triangle(const yo_geometry* g, const yo_prim* p, const ray_pre* r, float t_min, yo_hit* best) {
    if (p->mesh_primitive < 0 || p->mesh_primitive >= g->primitive_count || p->local_triangle < 0) return;
    const uint32_t base = g->prim_first_count[2 * p->mesh_primitive] + (uint32_t)p->local_triangle * 3u;
    if ((uint64_t)base + 2 >= (uint64_t)g->index_count) return;
    const uint32_t i0 = g->indices[base], i1 = g->indices[base + 1], i2 = g->indices[base + 2];
    if ((int64_t)i0 >= g->vertex_count || (int64_t)i1 >= g->vertex_count || (int64_t)i2 >= g->vertex_count) return;
    const float* p0 = vpos(g, i0);
    const float* p1 = vpos(g, i1);
    const float* p2 = vpos(g, i2);
    float e1[3], e2[3], pv[3], tv[3], qv[3];
    for (int a = 0; a < 3; ++a) {
        e1[a] = p1[a] - p0[a];
        e2[a] = p2[a] - p0[a];
    }
    cross3(r->d, e2, pv);
    const float det = dot3(e1, pv);
    if (fabsf(det) < 1.0e-8f) return;
    const float inv_det = 1.0f / det;
    for (int a = 0; a < 3; ++a) tv[a] = r->o[a] - p0[a];
    const float u = dot3(tv, pv) * inv_det;
    if (u < 0.0f || u > 1.0f) return;
    cross3(tv, e1, qv);
    const float v = dot3(r->d, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return;
    const float t = dot3(e2, qv) * inv_det;
    if (t <= t_min || t > best->t) return;
    if (t == best->t && best->hit && best->triangle_index >= 0 && p->flat_triangle_index >= best->triangle_index) return;
    best->hit = 1;
    best->t = t;
    best->triangle_index = p->flat_triangle_index;
    best->mesh_primitive = p->mesh_primitive;
    best->sphere = -1;
    best->u = u;
    best->v = v;
}

/* IntersectSphere + SphereNormal + SphereUv (src/geometry/intersection.cpp:108-151),
 * as used by IntersectAnalyticSphere (bvh_traversal.cpp:123-150). */
static int sphere_hit(const float* c, float radius, const ray_pre* r, float t_min, float t_max, float* t_out) {
    const float oc[3] = {r->o[0] - c[0], r->o[1] - c[1], r->o[2] - c[2]};
    const float a = dot3(r->d, r->d);
    const float b = 2.0f * dot3(oc, r->d);
    const float cc = dot3(oc, oc) - radius * radius;
    const float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return 0;
    const float sq = sqrtf(disc);
    const float inv_2a = 0.5f / a;
    const float t0 = (-b - sq) * inv_2a;
    if (t0 > t_min && t0 < t_max) {
        *t_out = t0;
        return 1;
    }
    const float t1 = (-b + sq) * inv_2a;
    if (t1 > t_min && t1 < t_max) {
        *t_out = t1;
        return 1;
    }
    return 0;
}

static void intersect_sphere(const yo_geometry* g, int32_t sphere, const ray_pre* r, float t_min, yo_hit* best,
                             int clear_instance) {
    if (sphere < 0 || sphere >= g->sphere_count) return;
    const float* s = g->spheres + 4 * sphere;
    float t;
    if (!sphere_hit(s, s[3], r, t_min, best->t, &t) || t >= best->t) return;
    float n[3];
    for (int a = 0; a < 3; ++a) n[a] = (r->o[a] + r->d[a] * t) - s[a];
    const float len = sqrtf(dot3(n, n));
    if (len > 0.0f) {
        for (int a = 0; a < 3; ++a) n[a] = n[a] / len;
    } else {
        n[0] = n[1] = n[2] = 0.0f;
    }
    const float pi = 3.14159265358979323846f;
    const float cy = n[1] < -1.0f ? -1.0f : (1.0f < n[1] ? 1.0f : n[1]);
    best->hit = 1;
    best->t = t;
    best->triangle_index = -1;
    best->mesh_primitive = -1;
    if (clear_instance) best->instance = -1;
    best->sphere = sphere;
    best->u = (atan2f(n[0], n[2]) + pi) / (2.0f * pi);
    best->v = (pi - acosf(cy)) / pi;
}

/* Growable traversal stack (the reference's TraversalStack, bvh_traversal.cpp:17-50). */
typedef struct stack_t_ {
    int32_t* node;
    float* entry;
    int64_t size, cap;
    int32_t inline_node[64];
    float inline_entry[64];
} trav_stack;

static void stack_init(trav_stack* s) {
    s->node = s->inline_node;
    s->entry = s->inline_entry;
    s->size = 0;
    s->cap = 64;
}

static void stack_push(trav_stack* s, int32_t node, float entry) {
    if (s->size == s->cap) {
        const int64_t cap = s->cap * 2;
        int32_t* n = (int32_t*)malloc((size_t)cap * sizeof(int32_t));
        float* e = (float*)malloc((size_t)cap * sizeof(float));
        memcpy(n, s->node, (size_t)s->size * sizeof(int32_t));
        memcpy(e, s->entry, (size_t)s->size * sizeof(float));
        if (s->node != s->inline_node) {
            free(s->node);
            free(s->entry);
        }
        s->node = n;
        s->entry = e;
        s->cap = cap;
    }
    s->node[s->size] = node;
    s->entry[s->size] = entry;
    ++s->size;
}

static void stack_free(trav_stack* s) {
    if (s->node != s->inline_node) {
        free(s->node);
        free(s->entry);
    }
}

/* IntersectBvh (bvh_traversal.cpp:253-345) on a precomputed ray. */
static yo_hit intersect_bvh_pre(const yo_geometry* g, const yo_bvh* bvh, const ray_pre* r, float t_min, float t_max,
                                yo_stats* st) {
    yo_hit best = miss_hit(t_max);
    if (bvh->node_count <= 0) return best;
    float root_entry = t_min;
    ++st->node_tests;
    if (!intersect_bounds(&bvh->nodes[0], r, t_min, best.t, &root_entry)) return best;
    trav_stack s;
    stack_init(&s);
    stack_push(&s, 0, root_entry);
    while (s.size > 0) {
        --s.size;
        const int32_t ni = s.node[s.size];
        const float ne = s.entry[s.size];
        if (ne > best.t) continue;
        if (ni < 0 || ni >= bvh->node_count) continue;
        const yo_node* node = &bvh->nodes[ni];
        if (node->primitive_count > 0) {
            for (int32_t i = node->payload_offset; i < node->payload_offset + node->primitive_count; ++i) {
                if (i < 0 || i >= bvh->primitive_index_count) continue;
                const int32_t pi = bvh->primitive_indices[i];
                if (pi < 0 || pi >= bvh->primitive_count) continue;
                const yo_prim* p = &bvh->primitives[pi];
                if (p->kind == 0) {
                    ++st->triangle_tests;
                    intersect_triangle(g, p, r, t_min, &best);
                } else {
                    ++st->sphere_tests;
                    intersect_sphere(g, p->sphere, r, t_min, &best, 0);
                }
            }
        } else {
            const int32_t li = ni + 1, ri = node->payload_offset;
            float le = t_min, re = t_min;
            int hl = 0, hr = 0;
            if (li >= 0 && li < bvh->node_count) {
                ++st->node_tests;
                hl = intersect_bounds(&bvh->nodes[li], r, t_min, best.t, &le);
            }
            if (ri >= 0 && ri < bvh->node_count) {
                ++st->node_tests;
                hr = intersect_bounds(&bvh->nodes[ri], r, t_min, best.t, &re);
            }
            if (hl && hr) {
                if (le <= re) {
                    stack_push(&s, ri, re);
                    stack_push(&s, li, le);
                } else {
                    stack_push(&s, li, le);
                    stack_push(&s, ri, re);
                }
            } else if (hl) {
                stack_push(&s, li, le);
            } else if (hr) {
                stack_push(&s, ri, re);
            }
        }
    }
    stack_free(&s);
    return best;
}

yo_hit yo_intersect_bvh(const yo_geometry* g, const yo_bvh* bvh, const float origin[3], const float dir[3],
                        float t_min, float t_max, yo_stats* stats) {
    ray_pre r;
    precompute(&r, origin, dir);
    return intersect_bvh_pre(g, bvh, &r, t_min, t_max, stats);
}

/* TransformPoint / TransformVector (src/core/transform.cpp:30-44). */
static void xform_point(const float* m, const float* p, float* o) {
    for (int r = 0; r < 3; ++r) o[r] = m[r] * p[0] + m[4 + r] * p[1] + m[8 + r] * p[2] + m[12 + r];
}
static void xform_vector(const float* m, const float* v, float* o) {
    for (int r = 0; r < 3; ++r) o[r] = m[r] * v[0] + m[4 + r] * v[1] + m[8 + r] * v[2];
}

/* IntersectTwoLevelBvh (src/accel/two_level_bvh.cpp:365-481). */
yo_hit yo_intersect_two_level(const yo_geometry* g, const yo_two_level* tl, const float origin[3],
                              const float dir[3], float t_min, float t_max, yo_stats* st) {
    yo_hit best = miss_hit(t_max);
    if (tl->tlas_node_count <= 0) return best;
    ray_pre r;
    precompute(&r, origin, dir);
    float root_entry = t_min;
    ++st->node_tests;
    if (!intersect_bounds(&tl->tlas_nodes[0], &r, t_min, best.t, &root_entry)) return best;
    trav_stack s;
    stack_init(&s);
    stack_push(&s, 0, root_entry);
    while (s.size > 0) {
        --s.size;
        const int32_t ni = s.node[s.size];
        const float ne = s.entry[s.size];
        if (ne > best.t) continue;
        if (ni < 0 || ni >= tl->tlas_node_count) continue;
        const yo_node* node = &tl->tlas_nodes[ni];
        if (node->primitive_count == 0) {
            const int32_t li = ni + 1, ri = node->payload_offset;
            float le = t_min, re = t_min;
            int hl = 0, hr = 0;
            if (li >= 0 && li < tl->tlas_node_count) {
                ++st->node_tests;
                hl = intersect_bounds(&tl->tlas_nodes[li], &r, t_min, best.t, &le);
            }
            if (ri >= 0 && ri < tl->tlas_node_count) {
                ++st->node_tests;
                hr = intersect_bounds(&tl->tlas_nodes[ri], &r, t_min, best.t, &re);
            }
            if (hl && hr) {
                if (le <= re) {
                    stack_push(&s, ri, re);
                    stack_push(&s, li, le);
                } else {
                    stack_push(&s, li, le);
                    stack_push(&s, ri, re);
                }
            } else if (hl) {
                stack_push(&s, li, le);
            } else if (hr) {
                stack_push(&s, ri, re);
            }
            continue;
        }
        for (int32_t i = node->payload_offset; i < node->payload_offset + node->primitive_count; ++i) {
            if (i < 0 || i >= tl->tlas_primitive_index_count) continue;
            const int32_t pi = tl->tlas_primitive_indices[i];
            if (pi < 0 || pi >= tl->tlas_primitive_count) continue;
            const int32_t* p = tl->tlas_primitives + 3 * pi;
            if (p[0] == 1) {
                ++st->sphere_tests;
                intersect_sphere(g, p[2], &r, t_min, &best, 1);
                continue;
            }
            const int32_t inst = p[1];
            if (inst < 0 || inst >= tl->instance_count) continue;
            const int32_t b = tl->instance_blas[inst];
            if (b < 0 || b >= tl->blas_count) continue;
            float oo[3], od[3];
            xform_point(tl->instance_w2o + 16 * inst, origin, oo);
            xform_vector(tl->instance_w2o + 16 * inst, dir, od);
            ray_pre orr;
            precompute(&orr, oo, od);
            yo_hit h = intersect_bvh_pre(g, &tl->blases[b], &orr, t_min, best.t, st);
            if (h.hit && h.t < best.t) {
                h.instance = inst;
                best = h;
            }
        }
    }
    stack_free(&s);
    return best;
}

/* ---------------------------------------------------------- batched drivers */

typedef struct trace_job {
    const yo_geometry* g;
    const yo_bvh* bvh;
    const yo_two_level* tl;
    const float* rays;
    int64_t n;
    yo_hit* hits;
    uint32_t *nt, *tt, *st;
    int worker, workers;
} trace_job;

static void* trace_worker(void* arg) {
    trace_job* j = (trace_job*)arg;
    for (int64_t i = j->worker; i < j->n; i += j->workers) {
        const float* r = j->rays + 8 * i;
        yo_stats s = {0, 0, 0};
        j->hits[i] = j->tl ? yo_intersect_two_level(j->g, j->tl, r, r + 4, r[3], r[7], &s)
                           : yo_intersect_bvh(j->g, j->bvh, r, r + 4, r[3], r[7], &s);
        if (j->nt) j->nt[i] = (uint32_t)s.node_tests;
        if (j->tt) j->tt[i] = (uint32_t)s.triangle_tests;
        if (j->st) j->st[i] = (uint32_t)s.sphere_tests;
    }
    return NULL;
}

static void run_trace(trace_job base, int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    trace_job jobs[256];
    for (int w = 0; w < threads; ++w) {
        jobs[w] = base;
        jobs[w].worker = w;
        jobs[w].workers = threads;
        if (threads == 1) {
            trace_worker(&jobs[w]);
        } else {
            pthread_create(&tid[w], NULL, trace_worker, &jobs[w]);
        }
    }
    if (threads > 1) {
        for (int w = 0; w < threads; ++w) pthread_join(tid[w], NULL);
    }
}

void yo_trace_flat(const yo_geometry* g, const yo_bvh* bvh, const float* rays, int64_t n, yo_hit* hits,
                   uint32_t* node_tests, uint32_t* tri_tests, uint32_t* sphere_tests, int threads) {
    trace_job j = {g, bvh, NULL, rays, n, hits, node_tests, tri_tests, sphere_tests, 0, 1};
    run_trace(j, threads);
}

void yo_trace_two_level(const yo_geometry* g, const yo_two_level* tl, const float* rays, int64_t n, yo_hit* hits,
                        uint32_t* node_tests, uint32_t* tri_tests, uint32_t* sphere_tests, int threads) {
    trace_job j = {g, NULL, tl, rays, n, hits, node_tests, tri_tests, sphere_tests, 0, 1};
    run_trace(j, threads);
}

/* IntersectAccelerationProbe (src/accel/acceleration.cpp:63-108) and
 * IntersectBvhProbe (bvh_traversal.cpp:347-391): iterated closest hit with a
 * cursor advanced by 1e-4 (1 + |t|), at most 4096 iterations, 64 hits. */
void yo_probe(const yo_geometry* g, const yo_bvh* flat, const yo_two_level* tl, const float* rays, int64_t n,
              const int32_t* targets, int32_t* counts, uint8_t* exhausted, yo_hit* hits) {
    for (int64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        const int32_t tp = targets[3 * i], ti = targets[3 * i + 1], ts = targets[3 * i + 2];
        int32_t count = 0;
        uint8_t ex = 0;
        float cursor = r[3];
        for (int iter = 0; iter < 4096; ++iter) {
            yo_stats st = {0, 0, 0};
            const yo_hit h = tl ? yo_intersect_two_level(g, tl, r, r + 4, cursor, r[7], &st)
                                : yo_intersect_bvh(g, flat, r, r + 4, cursor, r[7], &st);
            if (!h.hit) break;
            const int inst_ok = tl ? (ti < 0 || h.instance == ti) : 1;
            const int is_target = (tp >= 0 && h.triangle_index >= 0 && h.mesh_primitive == tp && inst_ok) ||
                                  (ts >= 0 && h.sphere == ts);
            if (is_target) {
                if (count < 64) {
                    hits[i * 64 + count++] = h;
                } else {
                    ex = 1;
                    break;
                }
            }
            float next = h.t + 1.0e-4f * (1.0f + fabsf(h.t));
            if (!(next > cursor)) next = cursor + 1.0e-4f;
            cursor = next;
            if (cursor >= r[7]) break;
        }
        counts[i] = count;
        exhausted[i] = ex;
    }
}

/* ------------------------------------------------------------------ sampler */

#define DEFAULT_SEED 0x9E3779B97F4A7C15ull

/* Mix64 / Mix32 / Hash32 (src/sampling/sampler.cpp:34-55): SplitMix64
 * finaliser and a 32-bit integer hash, combined per (seed, dim, lane). */
static uint64_t mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}

static uint32_t mix32(uint32_t v) {
    v ^= v >> 16;
    v *= 0x7FEB352Du;
    v ^= v >> 15;
    v *= 0x846CA68Bu;
    return v ^ (v >> 16);
}

static uint32_t hash32(uint64_t seed, uint32_t dim, int lane) {
    const uint64_t m = mix64(seed ^ ((uint64_t)dim * 0xD1B54A32D192ED03ull) ^
                             ((uint64_t)(uint32_t)lane * 0x94D049BB133111EBull));
    return mix32((uint32_t)m ^ (uint32_t)(m >> 32));
}

static float unit_float(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

static uint32_t reverse_bits(uint32_t v) {
    v = ((v & 0x55555555u) << 1) | ((v >> 1) & 0x55555555u);
    v = ((v & 0x33333333u) << 2) | ((v >> 2) & 0x33333333u);
    v = ((v & 0x0F0F0F0Fu) << 4) | ((v >> 4) & 0x0F0F0F0Fu);
    v = ((v & 0x00FF00FFu) << 8) | ((v >> 8) & 0x00FF00FFu);
    return (v << 16) | (v >> 16);
}

/* Sobol axes 0 and 1 (sampler.cpp:70-89): axis 0 is the bit reversal; axis 1
 * XORs direction numbers v_k = v_{k-1} ^ (v_{k-1} >> 1) from 0x80000000. */
static uint32_t sobol_bits(uint32_t index, int axis) {
    if (axis == 0) return reverse_bits(index);
    uint32_t value = 0, dirv = 0x80000000u;
    for (int bit = 0; bit < 32 && index; ++bit, dirv ^= dirv >> 1) {
        if (index & 1u) value ^= dirv;
        index >>= 1;
    }
    return value;
}

/* Laine-Karras nested-uniform scramble (sampler.cpp:94-102). */
static uint32_t owen_scramble(uint32_t v, uint32_t seed) {
    v = reverse_bits(v);
    v += seed;
    v ^= v * 0x6C50B47Cu;
    v ^= v * 0xB82F1E52u;
    v ^= v * 0xC7AFE638u;
    v ^= v * 0x8D22F6E6u;
    return reverse_bits(v);
}

static uint32_t spread_bits16(uint32_t v) {
    v &= 0x0000FFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

typedef struct sampler_t_ {
    int kind;
    uint64_t scene_seed, pixel_seed;
    uint32_t sobol_index;
    int sample_index, spp, bounce;
} sampler_state;

/* Sampler(kind, scene_seed, x, y, sample, spp, light_samples=1)
 * (sampler.cpp:138-166). */
static sampler_state make_sampler(int kind, uint64_t seed, int x, int y, int sample, int spp) {
    sampler_state s;
    s.kind = kind;
    s.scene_seed = seed;
    s.pixel_seed = mix64(seed ^ ((uint64_t)(uint32_t)x << 32) ^ (uint64_t)(uint32_t)y);
    s.sample_index = sample;
    s.spp = spp < 1 ? 1 : spp;
    s.bounce = 0;
    if (kind == 3) {
        unsigned c = 1;
        while (c < (unsigned)s.spp) c <<= 1;
        unsigned bits = 0;
        while ((1u << (bits + 1)) <= c) ++bits; /* bit_width(bit_ceil(spp)) - 1 */
        s.sobol_index = ((spread_bits16((uint32_t)x) | (spread_bits16((uint32_t)y) << 1)) << bits) | (uint32_t)sample;
    } else {
        s.sobol_index = (uint32_t)sample;
    }
    return s;
}

static float sample1d_at(const sampler_state* s, uint32_t dim, int lane) {
    if (s->kind == 2) return unit_float(owen_scramble(sobol_bits(s->sobol_index, 0), hash32(s->pixel_seed ^ DEFAULT_SEED, dim, lane)));
    if (s->kind == 3) return unit_float(owen_scramble(sobol_bits(s->sobol_index, 0), hash32(s->scene_seed, dim, lane)));
    return unit_float(hash32(s->pixel_seed ^ (uint64_t)(int64_t)s->sample_index, dim, lane));
}

static float clamp_unit(float v) {
    const float hi = nextafterf(1.0f, 0.0f);
    return v < 0.0f ? 0.0f : (hi < v ? hi : v);
}

/* Sample2DAt (sampler.cpp:194-229). */
static void sample2d_at(const sampler_state* s, uint32_t dim, int lane, float* out) {
    if (dim == 0 && s->spp == 1) {
        out[0] = 0.5f;
        out[1] = 0.5f;
        return;
    }
    if (s->kind == 1) {
        const int count = dim == 0 ? s->spp : 1;
        const int index = dim == 0 ? s->sample_index : lane;
        const int columns = (int)ceilf(sqrtf((float)count));
        const int rows = (count + columns - 1) / columns;
        const int ci = index < 0 ? 0 : (index > count - 1 ? count - 1 : index);
        const int cx = ci % columns, cy = ci / columns;
        out[0] = clamp_unit(((float)cx + sample1d_at(s, dim, lane)) / (float)columns);
        out[1] = clamp_unit(((float)cy + sample1d_at(s, dim + 1, lane)) / (float)rows);
        return;
    }
    if (s->kind == 2 || s->kind == 3) {
        const uint64_t seed = s->kind == 2 ? s->pixel_seed : s->scene_seed;
        out[0] = unit_float(owen_scramble(sobol_bits(s->sobol_index, 0), hash32(seed, dim, lane)));
        out[1] = unit_float(owen_scramble(sobol_bits(s->sobol_index, 1), hash32(seed, dim + 1, lane)));
        return;
    }
    out[0] = sample1d_at(s, dim, lane);
    out[1] = sample1d_at(s, dim + 1, lane);
}

void yo_sampler(int kind, uint64_t seed, int spp, const int32_t* q, int64_t n, int two_d, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        const int32_t* r = q + 6 * i;
        sampler_state s = make_sampler(kind, seed, r[0], r[1], r[2], spp);
        s.bounce = r[3] < 0 ? 0 : r[3];
        const uint32_t dim = r[4] == 0 ? 0u : (uint32_t)r[4] + (uint32_t)s.bounce * 16u; /* AbsoluteDimension */
        if (two_d) sample2d_at(&s, dim, r[5], out + 2 * i);
        else out[i] = sample1d_at(&s, dim, r[5]);
    }
}

/* SeedForPixelSample (sampler.cpp:304-310). */
uint64_t yo_seed_for_pixel_sample(uint64_t seed, int x, int y, int sample) {
    uint64_t v = mix64(seed);
    v ^= mix64((uint64_t)(int64_t)x + 0xA24BAED4963EE407ull);
    v ^= mix64((uint64_t)(int64_t)y + 0x9FB21C651E98DF25ull);
    v ^= mix64((uint64_t)(int64_t)sample + 0xC2B2AE3D27D4EB4Full);
    return mix64(v);
}

/* PCG32 (include/yaoray/core/rng.hpp:15-48; O'Neill 2014, XSH-RR output). */
void yo_rng_floats(uint64_t seed, int count, float* out) {
    uint64_t state = 0, inc = (seed << 1u) | 1u;
#define PCG_STEP(res)                                                          \
    do {                                                                       \
        const uint64_t old = state;                                            \
        state = old * 6364136223846793005ull + inc;                            \
        const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);           \
        const uint32_t rot = (uint32_t)(old >> 59u);                           \
        res = (xs >> rot) | (xs << ((0u - rot) & 31u));                        \
    } while (0)
    uint32_t dummy;
    PCG_STEP(dummy);
    state += seed;
    PCG_STEP(dummy);
    (void)dummy;
    for (int i = 0; i < count; ++i) {
        uint32_t v;
        PCG_STEP(v);
        out[i] = (float)(v >> 8) * (1.0f / 16777216.0f);
    }
#undef PCG_STEP
}

/* ------------------------------------------------------------------- camera */

/* PerspectiveDirection (src/scene/camera.cpp:9-16): vertical fov, aspect W/H,
 * film y pointing down, normalised. */
static void persp_dir(const float* cam, float w, float h, float fx, float fy, float* out) {
    const float aspect = w / h;
    const float half_h = tanf(cam[12] * 0.5f);
    const float sx = (2.0f * fx / w - 1.0f) * aspect * half_h;
    const float sy = (1.0f - 2.0f * fy / h) * half_h;
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = cam[3 + a] + cam[6 + a] * sx + cam[9 + a] * sy;
    const float len = sqrtf(dot3(d, d));
    for (int a = 0; a < 3; ++a) out[a] = len > 0.0f ? d[a] / len : 0.0f;
}

void yo_camera_rays(const float* camera, int width, int height, const int32_t* pixels, const float* samples,
                    int64_t n, float* out) {
    const float w = (float)(width < 1 ? 1 : width);
    const float h = (float)(height < 1 ? 1 : height);
    for (int64_t i = 0; i < n; ++i) {
        const float fx = (float)pixels[2 * i] + samples[2 * i];
        const float fy = (float)pixels[2 * i + 1] + samples[2 * i + 1];
        out[6 * i + 0] = camera[0];
        out[6 * i + 1] = camera[1];
        out[6 * i + 2] = camera[2];
        persp_dir(camera, w, h, fx, fy, out + 6 * i + 3);
    }
}

/* --------------------------------------------------------------------- film */

typedef struct film_px {
    float sum[3];
    uint32_t samples;
    float mean, m2;
    float albedo[3];
    float normal[3];
    float depth;
    uint32_t aov_samples;
} film_px;

/* Film::AddSample (src/film/film.cpp:160-183): non-finite beauty is counted
 * and dropped; Welford update of the luminance (Rec.709 weights); AOVs only
 * for finite primary hits with depth >= 0. */
uint64_t yo_film_accumulate(int width, int height, const float* samples, int64_t n, void* pixels_out) {
    film_px* px = (film_px*)pixels_out;
    memset(px, 0, (size_t)width * (size_t)height * sizeof(film_px));
    uint64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        const float* s = samples + 13 * i;
        const int x = (int)s[0], y = (int)s[1];
        if (x < 0 || y < 0 || x >= width || y >= height) continue;
        if (!isfinite(s[2]) || !isfinite(s[3]) || !isfinite(s[4])) {
            ++bad;
            continue;
        }
        film_px* p = &px[(size_t)y * (size_t)width + (size_t)x];
        for (int a = 0; a < 3; ++a) p->sum[a] = p->sum[a] + s[2 + a];
        ++p->samples;
        const float lum = 0.2126f * s[2] + 0.7152f * s[3] + 0.0722f * s[4];
        const float delta = lum - p->mean;
        p->mean += delta / (float)p->samples;
        const float delta2 = lum - p->mean;
        p->m2 += delta * delta2;
        const int primary = s[12] != 0.0f;
        if (primary && isfinite(s[5]) && isfinite(s[6]) && isfinite(s[7]) && isfinite(s[8]) && isfinite(s[9]) &&
            isfinite(s[10]) && isfinite(s[11]) && s[11] >= 0.0f) {
            for (int a = 0; a < 3; ++a) {
                p->albedo[a] = p->albedo[a] + s[5 + a];
                p->normal[a] = p->normal[a] + s[8 + a];
            }
            p->depth += s[11];
            ++p->aov_samples;
        }
    }
    return bad;
}

/* ----------------------------------------------------------------- texture */

/* RenderTexture sampling (src/shading/texture.cpp:14-322). A texture is the
 * image plus its mip chain, levels stored one after the other. */
typedef struct tex_level {
    int w, h;
    const float* t; /* RGBA rows */
} tex_level;

typedef struct tex_view {
    int width, height, filter, wrap_s, wrap_t, levels;
    tex_level lv[40];
} tex_view;

typedef struct rgba {
    float x, y, z, w;
} rgba;

static rgba rgba_black(void) { rgba c = {0.0f, 0.0f, 0.0f, 1.0f}; return c; } /* Color4f{} */
static rgba rgba_add(rgba a, rgba b) { rgba c = {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; return c; }
static rgba rgba_scale(rgba a, float s) { rgba c = {a.x * s, a.y * s, a.z * s, a.w * s}; return c; }
static rgba rgba_div(rgba a, float s) { rgba c = {a.x / s, a.y / s, a.z / s, a.w / s}; return c; }
/* Lerp (texture.cpp:101-103). */
static rgba rgba_lerp(rgba a, rgba b, float t) { return rgba_add(rgba_scale(a, 1.0f - t), rgba_scale(b, t)); }
static float fmax_std(float a, float b) { return a < b ? b : a; }
static float fmin_std(float a, float b) { return b < a ? b : a; }
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }

/* ApplyWrap (texture.cpp:20-28): 0 repeat, 1 clamp, 2 mirrored repeat. */
static float apply_wrap(float v, int wrap) {
    if (wrap == 1) return v < 0.0f ? 0.0f : (1.0f < v ? 1.0f : v);
    const float base = floorf(v);
    const float fraction = v - base;
    if (wrap == 2) return (((int)base) & 1) == 0 ? fraction : 1.0f - fraction;
    return fraction < 0.0f ? fraction + 1.0f : fraction;
}

/* WrappedTexelIndex (texture.cpp:30-40). */
static int wrapped_index(int value, int count, int wrap) {
    if (wrap == 1) return clampi(value, 0, count - 1);
    if (wrap == 2) {
        const int period = count * 2;
        int w = value % period;
        if (w < 0) w += period;
        return w < count ? w : period - 1 - w;
    }
    int w = value % count;
    if (w < 0) w += count;
    return w;
}

/* TexelAt (texture.cpp:90-99). */
static rgba texel_at(tex_level l, int x, int y, int ws, int wt) {
    if (l.w <= 0 || l.h <= 0 || !l.t) return rgba_black();
    const int ix = wrapped_index(x, l.w, ws), iy = wrapped_index(y, l.h, wt);
    const float* p = l.t + 4 * ((int64_t)iy * l.w + ix);
    rgba c = {p[0], p[1], p[2], p[3]};
    return c;
}

/* Level (texture.cpp:42-60). */
static tex_level tex_level_of(const tex_view* t, int level) {
    const int i = level <= 0 ? 0 : (level < t->levels - 1 ? level : t->levels - 1);
    return t->lv[i];
}

/* SampleNearest (texture.cpp:105-113). */
static rgba sample_nearest(tex_level l, const tex_view* t, float u, float v) {
    if (l.w <= 0 || l.h <= 0 || !l.t) return rgba_black();
    const int x = clampi((int)floorf(apply_wrap(u, t->wrap_s) * (float)l.w), 0, l.w - 1);
    const int y = clampi((int)floorf(apply_wrap(v, t->wrap_t) * (float)l.h), 0, l.h - 1);
    return texel_at(l, x, y, t->wrap_s, t->wrap_t);
}

/* SampleBilinear (texture.cpp:115-130). */
static rgba sample_bilinear(tex_level l, const tex_view* t, float u, float v) {
    if (l.w <= 0 || l.h <= 0 || !l.t) return rgba_black();
    if (l.w == 1 && l.h == 1) {
        rgba c = {l.t[0], l.t[1], l.t[2], l.t[3]};
        return c;
    }
    const float s = apply_wrap(u, t->wrap_s) * (float)l.w - 0.5f;
    const float tt = apply_wrap(v, t->wrap_t) * (float)l.h - 0.5f;
    const int s0 = (int)floorf(s), t0 = (int)floorf(tt);
    const float ds = s - (float)s0, dt = tt - (float)t0;
    const rgba c00 = texel_at(l, s0, t0, t->wrap_s, t->wrap_t);
    const rgba c10 = texel_at(l, s0 + 1, t0, t->wrap_s, t->wrap_t);
    const rgba c01 = texel_at(l, s0, t0 + 1, t->wrap_s, t->wrap_t);
    const rgba c11 = texel_at(l, s0 + 1, t0 + 1, t->wrap_s, t->wrap_t);
    return rgba_lerp(rgba_lerp(c00, c10, ds), rgba_lerp(c01, c11, ds), dt);
}

/* LodForFootprint (texture.cpp:132-138). */
static float lod_for_footprint(const tex_view* t, const float* f) {
    const float w = (float)(t->width > 1 ? t->width : 1), h = (float)(t->height > 1 ? t->height : 1);
    const float dx = hypotf(f[0] * w, f[1] * h);
    const float dy = hypotf(f[2] * w, f[3] * h);
    return fmax_std(0.0f, log2f(fmax_std(1.0f, fmax_std(dx, dy))));
}

/* EwaWeights (texture.cpp:140-152). */
static float ewa_weight(size_t i) {
    static float weights[128];
    static int ready = 0;
    if (!ready) {
        const float alpha = 2.0f, edge = expf(-alpha);
        for (size_t k = 0; k < 128; ++k) {
            const float r2 = (float)k / (float)(128 - 1);
            weights[k] = expf(-alpha * r2) - edge;
        }
        ready = 1;
    }
    return weights[i];
}

/* SampleEwaLevel (texture.cpp:154-213). */
static rgba sample_ewa_level(const tex_view* t, float u, float v, const float* f, int level) {
    const tex_level l = tex_level_of(t, level);
    if (l.w <= 0 || l.h <= 0 || !l.t) return rgba_black();
    float dsdx = f[0] * (float)l.w, dtdx = f[1] * (float)l.h;
    float dsdy = f[2] * (float)l.w, dtdy = f[3] * (float)l.h;
    if (dsdx * dsdx + dtdx * dtdx < dsdy * dsdy + dtdy * dtdy) {
        float tmp = dsdx; dsdx = dsdy; dsdy = tmp;
        tmp = dtdx; dtdx = dtdy; dtdy = tmp;
    }
    const float major = hypotf(dsdx, dtdx);
    float minor = hypotf(dsdy, dtdy);
    const float max_anisotropy = 8.0f;
    if (minor > 0.0f && major > minor * max_anisotropy) {
        const float scale = major / (minor * max_anisotropy);
        dsdy *= scale;
        dtdy *= scale;
        minor *= scale;
    }
    if (minor == 0.0f) return sample_bilinear(l, t, u, v);
    const float s = apply_wrap(u, t->wrap_s) * (float)l.w - 0.5f;
    const float tc = apply_wrap(v, t->wrap_t) * (float)l.h - 0.5f;
    float a = dtdx * dtdx + dtdy * dtdy + 1.0f;
    float b = -2.0f * (dsdx * dtdx + dsdy * dtdy);
    float c = dsdx * dsdx + dsdy * dsdy + 1.0f;
    const float inverse = 1.0f / (a * c - 0.25f * b * b);
    a *= inverse;
    b *= inverse;
    c *= inverse;
    const float determinant = -b * b + 4.0f * a * c;
    if (determinant <= 0.0f) return sample_bilinear(l, t, u, v);
    const float inverse_det = 1.0f / determinant;
    const float radius_s = 2.0f * sqrtf(c * inverse_det);
    const float radius_t = 2.0f * sqrtf(a * inverse_det);
    const int s0 = (int)ceilf(s - radius_s), s1 = (int)floorf(s + radius_s);
    const int t0 = (int)ceilf(tc - radius_t), t1 = (int)floorf(tc + radius_t);
    rgba sum = rgba_black();
    float weight_sum = 0.0f;
    for (int it = t0; it <= t1; ++it) {
        for (int is = s0; is <= s1; ++is) {
            const float ss = (float)is - s, tt = (float)it - tc;
            const float r2 = a * ss * ss + b * ss * tt + c * tt * tt;
            if (r2 >= 1.0f) continue;
            size_t wi = (size_t)(r2 * 128.0f);
            if (wi > 127) wi = 127;
            const float weight = ewa_weight(wi);
            sum = rgba_add(sum, rgba_scale(texel_at(l, is, it, t->wrap_s, t->wrap_t), weight));
            weight_sum += weight;
        }
    }
    return weight_sum > 0.0f ? rgba_div(sum, weight_sum) : sample_bilinear(l, t, u, v);
}

/* SampleTrilinear (texture.cpp:215-223). */
static rgba sample_trilinear(const tex_view* t, float u, float v, const float* f) {
    const float lod = fmin_std(lod_for_footprint(t, f), (float)(t->levels - 1));
    const int l0 = (int)floorf(lod);
    const int l1 = l0 + 1 < t->levels - 1 ? l0 + 1 : t->levels - 1;
    return rgba_lerp(sample_bilinear(tex_level_of(t, l0), t, u, v), sample_bilinear(tex_level_of(t, l1), t, u, v),
                     lod - (float)l0);
}

/* SampleEwa (texture.cpp:225-238). */
static rgba sample_ewa(const tex_view* t, float u, float v, const float* f) {
    const float w = (float)(t->width > 1 ? t->width : 1), h = (float)(t->height > 1 ? t->height : 1);
    const float dx = hypotf(f[0] * w, f[1] * h);
    const float dy = hypotf(f[2] * w, f[3] * h);
    const float minor = fmax_std(1.0f, fmin_std(dx, dy));
    const float lod = fmin_std(fmax_std(0.0f, log2f(minor)), (float)(t->levels - 1));
    const int l0 = (int)floorf(lod);
    const int l1 = l0 + 1 < t->levels - 1 ? l0 + 1 : t->levels - 1;
    return rgba_lerp(sample_ewa_level(t, u, v, f, l0), sample_ewa_level(t, u, v, f, l1), lod - (float)l0);
}

/* BuildTextureMipChain (texture.cpp:242-264): level dims halve with
 * round-up; each texel is ((a + b) + c) + d of the 2x2 block, times 0.25.
 * Writes the levels after the image into `out`; returns their count. */
int yo_texture_mip_chain(int width, int height, const float* texels, int wrap_s, int wrap_t, float* out, int32_t* dims) {
    if (width <= 0 || height <= 0 || !texels) return 0;
    tex_level src = {width, height, texels};
    int count = 0;
    float* dst = out;
    while (src.w > 1 || src.h > 1) {
        const int w = (src.w + 1) / 2 > 1 ? (src.w + 1) / 2 : 1;
        const int h = (src.h + 1) / 2 > 1 ? (src.h + 1) / 2 : 1;
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                rgba f = texel_at(src, x * 2, y * 2, wrap_s, wrap_t);
                f = rgba_add(f, texel_at(src, x * 2 + 1, y * 2, wrap_s, wrap_t));
                f = rgba_add(f, texel_at(src, x * 2, y * 2 + 1, wrap_s, wrap_t));
                f = rgba_add(f, texel_at(src, x * 2 + 1, y * 2 + 1, wrap_s, wrap_t));
                f = rgba_scale(f, 0.25f);
                float* p = dst + 4 * ((int64_t)y * w + x);
                p[0] = f.x; p[1] = f.y; p[2] = f.z; p[3] = f.w;
            }
        }
        dims[2 * count] = w;
        dims[2 * count + 1] = h;
        ++count;
        src.w = w;
        src.h = h;
        src.t = dst;
        dst += 4 * (int64_t)w * h;
    }
    return count;
}

/* SampleTexture4 (texture.cpp:297-309) after BuildTextureMipChain. */
void yo_texture_sample(int width, int height, const float* texels, int filter, int wrap_s, int wrap_t,
                       const float* uvs, const float* footprints, int64_t n, float* out) {
    tex_view t;
    memset(&t, 0, sizeof t);
    t.width = width;
    t.height = height;
    t.filter = filter;
    t.wrap_s = wrap_s;
    t.wrap_t = wrap_t;
    float* chain = NULL;
    if (width > 0 && height > 0 && texels) {
        chain = (float*)malloc(sizeof(float) * 4 * ((size_t)width * height + 64));
        int32_t dims[80];
        const int mips = yo_texture_mip_chain(width, height, texels, wrap_s, wrap_t, chain, dims);
        t.levels = 1 + mips;
        t.lv[0].w = width;
        t.lv[0].h = height;
        t.lv[0].t = texels;
        const float* at = chain;
        for (int l = 0; l < mips; ++l) {
            t.lv[1 + l].w = dims[2 * l];
            t.lv[1 + l].h = dims[2 * l + 1];
            t.lv[1 + l].t = at;
            at += 4 * (int64_t)dims[2 * l] * dims[2 * l + 1];
        }
    }
    static const float zero[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int64_t i = 0; i < n; ++i) {
        const float u = uvs[2 * i], v = uvs[2 * i + 1];
        const float* f = footprints ? footprints + 4 * i : zero;
        const int fzero = f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f;
        rgba c;
        if (t.width <= 0 || t.height <= 0 || t.levels == 0) c = rgba_black();
        else if (t.filter == 0) c = sample_nearest(t.lv[0], &t, u, v);
        else if (t.filter == 2 && !fzero && t.levels > 1) c = sample_trilinear(&t, u, v, f);
        else if (t.filter == 3 && !fzero && t.levels > 1) c = sample_ewa(&t, u, v, f);
        else c = sample_bilinear(t.lv[0], &t, u, v);
        out[4 * i] = c.x;
        out[4 * i + 1] = c.y;
        out[4 * i + 2] = c.z;
        out[4 * i + 3] = c.w;
    }
    free(chain);
}
