/*
 * rtpg_oracle.c -- CPU restatement of RTLib's path-guiding hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA kernels of rtlib_b200: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  The product
 * never calls it and has no CPU fallback.
 *
 * Parity is pinned: tests/test_oracle_vs_reference.py checks this restatement against
 * RTLib's OWN code compiled on the host (oracle/ref, built into oracle/_ref) on identical
 * seeded inputs -- topology bit-exact, sums and pdfs within float-rounding tolerance
 * (RTLib sums in float, this restatement in 64-bit fixed point).
 *
 * It restates, with the same float expression order as the reference:
 *   SD-tree      OPX7UtilsPathGuiding.h (PG.h below)
 *     spatial descent   STreeT::GetDTreeWrapper / STreeNodeT::GetChildIdx   PG.h:639-648,546-569
 *     record            DTreeWrapperT::Record -> DTreeT::Impl<Nearest>::RecordIrradiance
 *                       -> DTreeNodeT::Record                                PG.h:514-520,417-428,113-125
 *     build             RTDTreeT::Build / DTreeNodeT::Build,GetArea          PG.h:948-957,356-369,342-355
 *     spatial refine    RTSTreeT::Refine / SubDivide / ShallSplit            PG.h:1275-1311,1231-1247,1270-1274
 *     quadtree reset    RTDTreeT::Reset                                      PG.h:888-947
 *     sample / pdf      DTreeT::Sample,Pdf,GetMean / DTreeNodeT::Sample,Pdf  PG.h:478-490,447-451,229-320
 *   math / rng   Xorshift32 (Random.h:37-51), to_uniform_float (Math.h:682-694),
 *                dir_to_canonical / canonical_to_dir (VectorFunction.h:5698-5720), pcg1d (Hash.h:13-18)
 *   hash grid    DoubleBufferedHashGrid3T FindFromCur / FindFromPrv           OPX7UtilsGrid.h:157-353
 *   Morton tree  MortonQuadTreeT Record / SampleAndPdf / Pdf, Morton2Utils    OPX7UtilsMorton.h:39-449
 *                mortonBuildKernel pyramid                                    OPX7UtilsMortonBuild.cu:2-16
 *
 * The two deliberate differences from the reference are the ones the CUDA path makes:
 *   1. sums are accumulated as int64 fixed point (value * 2^frac_bits, round to nearest)
 *      so that they do not depend on record order; they become float when a tree is built;
 *   2. quadtree nodes are numbered breadth first (the reference numbers them depth first,
 *      last child first); export_* write a canonical pre-order stream so topologies compare
 *      independently of numbering.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O_INV_2PI ((float)0.15915494309189533576888376337251436203445964574046)
#define O_2PI ((float)6.283185307179586476925286766559)

/* ------------------------------------------------------------------ rng / math */
static inline uint32_t xs32_next(uint32_t* s) {
    uint32_t y = *s;
    y = y ^ (y << 13);
    y = y ^ (y >> 17);
    return *s = y ^ (y << 5);
}
static inline float to_uniform_float(uint32_t v) {
    uint32_t b = (v >> 9) | (0x7Fu << 23);
    float f;
    memcpy(&f, &b, 4);
    return f - 1.0f;
}
static inline float rnd1(uint32_t* s) { return to_uniform_float(xs32_next(s)); }

uint32_t or_pcg1d(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

void or_dir_to_canonical(int64_t n, const float* d, float* uv) {
    for (int64_t i = 0; i < n; ++i) {
        float x = d[3 * i], y = d[3 * i + 1], z = d[3 * i + 2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) { uv[2 * i] = 0.0f; uv[2 * i + 1] = 0.0f; continue; }
        z = z < -1.0f ? -1.0f : (z > 1.0f ? 1.0f : z);
        float phi = atan2f(y, x);
        while (phi < 0.0f) phi += O_2PI;
        uv[2 * i] = (z + 1.0f) / 2.0f;
        uv[2 * i + 1] = phi * O_INV_2PI;
    }
}
static void canonical_to_dir(float u, float v, float* out) {
    const float cosTheta = 2.0f * u - 1.0f;
    const float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
    const float phi = O_2PI * v;
    out[0] = sinTheta * cosf(phi);
    out[1] = sinTheta * sinf(phi);
    out[2] = cosTheta;
}
static void normalize3(float* v) {
    float l = sqrtf((v[0] * v[0]) + (v[1] * v[1]) + (v[2] * v[2]));
    v[0] /= l; v[1] /= l; v[2] /= l;
}

/* fixed point: round-to-nearest of v * 2^bits, saturated */
static inline int64_t to_fx(float v, int bits, uint32_t* status) {
    float s = ldexpf(v, bits);
    if (!(s < 9.2233720368547758e18f)) { *status |= 1u; return INT64_MAX; }
    return llrintf(s);
}
static inline float fx_to_float(int64_t x, int bits) { return ldexpf((float)x, -bits); }

/* ------------------------------------------------------------------ SD-tree */
typedef struct { uint32_t c[4]; } OChild; /* local child index, 0 = leaf */

typedef struct {
    /* building tree */
    uint32_t nb;
    OChild* bch;
    int64_t* bsum; /* 4 per node */
    int64_t bstatw;
    float bstatw_f; /* building stat-weight as the reference would hold it during Refine */
    /* sampling tree */
    uint32_t ns;
    OChild* sch;
    float* ssum;
    float s_sum, s_area, s_statw;
    int max_depth_seen;
} ODTree;

typedef struct {
    int32_t child0; /* first child (children are child0, child0+1); -1 for a leaf */
    int32_t dtree;  /* leaf: dtree index */
} OSNode;

typedef struct {
    float mn[3], mx[3];
    int frac_bits;
    int max_dtree_depth;
    float subdiv_th;
    uint32_t node_cap;
    OSNode* st;
    uint32_t nst, capst;
    ODTree* dt;
    uint32_t ndt, capdt;
    uint32_t status;
} OSDTree;

static void dtree_init_single(ODTree* d) {
    memset(d, 0, sizeof(*d));
    d->nb = 1;
    d->bch = (OChild*)calloc(1, sizeof(OChild));
    d->bsum = (int64_t*)calloc(4, sizeof(int64_t));
    d->ns = 1;
    d->sch = (OChild*)calloc(1, sizeof(OChild));
    d->ssum = (float*)calloc(4, sizeof(float));
}
static void dtree_free(ODTree* d) { free(d->bch); free(d->bsum); free(d->sch); free(d->ssum); }

static uint32_t add_dtree(OSDTree* t) {
    if (t->ndt == t->capdt) {
        t->capdt = t->capdt ? 2 * t->capdt : 64;
        t->dt = (ODTree*)realloc(t->dt, sizeof(ODTree) * t->capdt);
    }
    return t->ndt++;
}
static uint32_t add_snodes(OSDTree* t, uint32_t k) {
    while (t->nst + k > t->capst) {
        t->capst = t->capst ? 2 * t->capst : 256;
        t->st = (OSNode*)realloc(t->st, sizeof(OSNode) * t->capst);
    }
    uint32_t r = t->nst;
    t->nst += k;
    return r;
}

/* RTSTreeT constructor (PG.h:1211-1217): the AABB is cubified to its largest extent. */
void* or_sdtree_new(const float* mn, const float* mx, int max_dtree_depth, float subdiv_th, int frac_bits,
                    uint32_t node_cap) {
    OSDTree* t = (OSDTree*)calloc(1, sizeof(OSDTree));
    float size[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    float m = size[0] > size[1] ? size[0] : size[1];
    m = m > size[2] ? m : size[2];
    for (int k = 0; k < 3; ++k) { t->mn[k] = mn[k]; t->mx[k] = mn[k] + m; }
    t->frac_bits = frac_bits;
    t->max_dtree_depth = max_dtree_depth;
    t->subdiv_th = subdiv_th;
    t->node_cap = node_cap;
    uint32_t r = add_snodes(t, 1);
    uint32_t d = add_dtree(t);
    dtree_init_single(&t->dt[d]);
    t->st[r].child0 = -1;
    t->st[r].dtree = (int32_t)d;
    return t;
}
void or_sdtree_free(void* h) {
    OSDTree* t = (OSDTree*)h;
    for (uint32_t i = 0; i < t->ndt; ++i) dtree_free(&t->dt[i]);
    free(t->dt); free(t->st); free(t);
}
uint32_t or_sdtree_status(void* h) { return ((OSDTree*)h)->status; }

/* STreeT::GetDTreeWrapper (PG.h:639-648) + STreeNodeT::GetChildIdx (PG.h:546-552).
 * The axis of a node is its depth mod 3 (root 0, SubDivide gives children (axis+1)%3,
 * PG.h:1240).  The child index int(2p) is clamped to [0,1] so that p == 1 or positions
 * outside the AABB stay in bounds (the reference would index out of range there). */
static int32_t leaf_dtree(const OSDTree* t, const float* pos) {
    float size[3] = {t->mx[0] - t->mn[0], t->mx[1] - t->mn[1], t->mx[2] - t->mn[2]};
    float p[3];
    for (int k = 0; k < 3; ++k) p[k] = (pos[k] - t->mn[k]) / size[k];
    uint32_t n = 0;
    int axis = 0;
    while (t->st[n].child0 >= 0) {
        float v = p[axis] * 2.0f;
        int idx = (int)v;
        idx = idx < 0 ? 0 : (idx > 1 ? 1 : idx);
        p[axis] = v - (float)idx;
        n = (uint32_t)t->st[n].child0 + (uint32_t)idx;
        axis = axis == 2 ? 0 : axis + 1;
    }
    return t->st[n].dtree;
}

/* DTreeNodeT::GetChildIdx (PG.h:69-82). */
static inline int quad_child(float* p) {
    int r = 0;
    for (int i = 0; i < 2; ++i) {
        if (p[i] < 0.5f) p[i] *= 2.0f;
        else { p[i] = 2.0f * p[i] - 1.0f; r |= 1 << i; }
    }
    return r;
}

/* DTreeWrapperT::Record (PG.h:514-520) -> Impl<Nearest>::RecordIrradiance (PG.h:417-428)
 * -> DTreeNodeT::Record (PG.h:113-125), with fixed-point accumulation. */
void or_sdtree_record(void* h, int64_t n, const float* pos, const float* uv, const float* radiance,
                      const float* wo_pdf, const float* stat_w, const uint8_t* is_delta) {
    OSDTree* t = (OSDTree*)h;
    for (int64_t i = 0; i < n; ++i) {
        if (is_delta && is_delta[i]) continue;
        const float wo = wo_pdf ? wo_pdf[i] : 1.0f;
        const float sw = stat_w ? stat_w[i] : 1.0f;
        const float irr = radiance[i] / wo;
        ODTree* d = &t->dt[leaf_dtree(t, pos + 3 * i)];
        if (!(isfinite(sw) && sw > 0.0f)) continue;
        d->bstatw += to_fx(sw, t->frac_bits, &t->status);
        if (!(isfinite(irr) && irr > 0.0f)) continue;
        const float v = irr * sw;
        float p[2] = {uv[2 * i], uv[2 * i + 1]};
        uint32_t cur = 0;
        int idx = quad_child(p);
        while (d->bch[cur].c[idx] != 0) {
            cur = d->bch[cur].c[idx];
            idx = quad_child(p);
        }
        d->bsum[4 * cur + idx] += to_fx(v, t->frac_bits, &t->status);
    }
}

/* RTDTreeT::Build (PG.h:948-957): bottom-up sums (nodes are breadth-first, so every child
 * has a larger index than its parent), area (DTreeNodeT::GetArea, PG.h:342-355) in the same
 * float order, root sum, then RTDTreeWrapperT::Build's "sampling = building" (PG.h:1086-1090). */
static void dtree_build(ODTree* d, int bits) {
    for (int64_t n = (int64_t)d->nb - 1; n >= 0; --n) {
        for (int i = 0; i < 4; ++i) {
            uint32_t c = d->bch[n].c[i];
            if (c) d->bsum[4 * n + i] = d->bsum[4 * c] + d->bsum[4 * c + 1] + d->bsum[4 * c + 2] + d->bsum[4 * c + 3];
        }
    }
    free(d->sch); free(d->ssum);
    d->ns = d->nb;
    d->sch = (OChild*)malloc(sizeof(OChild) * d->nb);
    d->ssum = (float*)malloc(sizeof(float) * 4 * d->nb);
    memcpy(d->sch, d->bch, sizeof(OChild) * d->nb);
    for (uint32_t k = 0; k < 4 * d->nb; ++k) d->ssum[k] = fx_to_float(d->bsum[k], bits);
    float* area = (float*)malloc(sizeof(float) * d->nb);
    for (int64_t n = (int64_t)d->nb - 1; n >= 0; --n) {
        float a = 0.0f;
        for (int i = 0; i < 4; ++i) {
            if (d->ssum[4 * n + i] > 0.0f) {
                uint32_t c = d->sch[n].c[i];
                if (!c) a += 1.0f / 4.0f;
                else a += area[c] / 4.0f;
            }
        }
        area[n] = a;
    }
    d->s_area = area[0];
    free(area);
    float s = 0.0f;
    for (int i = 0; i < 4; ++i) s += d->ssum[i];
    d->s_sum = s;
    d->s_statw = fx_to_float(d->bstatw, bits);
    d->bstatw_f = d->s_statw;
}
void or_sdtree_build(void* h) {
    OSDTree* t = (OSDTree*)h;
    for (uint32_t i = 0; i < t->ndt; ++i) dtree_build(&t->dt[i], t->frac_bits);
}

/* RTDTreeT::Reset (PG.h:888-947), breadth first.  A node either mirrors a node of the
 * previous (sampling) tree, or -- below a previous leaf quadrant -- is a "copy of itself"
 * whose four sums are the parent quadrant's sum / 4 (PG.h:926-933). */
typedef struct { uint32_t src; float vsum; int depth; } OSrc; /* src == UINT32_MAX: virtual */

static void dtree_reset(ODTree* d, int max_depth, float th, uint32_t cap, uint32_t* status) {
    const float total = d->s_sum;
    uint32_t capn = 64, nn = 1;
    OChild* ch = (OChild*)calloc(capn, sizeof(OChild));
    OSrc* src = (OSrc*)malloc(sizeof(OSrc) * capn);
    src[0].src = 0; src[0].vsum = 0.0f; src[0].depth = 1;
    int maxd = 0;
    int full = 0;
    for (uint32_t n = 0; n < nn && !full; ++n) {
        const OSrc s = src[n];
        if (s.depth > maxd) maxd = s.depth;
        for (int i = 0; i < 4; ++i) {
            const float si = s.src != UINT32_MAX ? d->ssum[4 * s.src + i] : s.vsum;
            const float fraction = total > 0.0f ? si / total : powf(0.25f, (float)s.depth);
            if (s.depth < max_depth && fraction > th) {
                if (nn == cap) { *status |= 2u; full = 1; break; }
                if (nn == capn) {
                    capn *= 2;
                    ch = (OChild*)realloc(ch, sizeof(OChild) * capn);
                    src = (OSrc*)realloc(src, sizeof(OSrc) * capn);
                }
                memset(&ch[nn], 0, sizeof(OChild));
                if (s.src != UINT32_MAX && d->sch[s.src].c[i] != 0) { src[nn].src = d->sch[s.src].c[i]; src[nn].vsum = 0.0f; }
                else { src[nn].src = UINT32_MAX; src[nn].vsum = si / 4.0f; }
                src[nn].depth = s.depth + 1;
                ch[n].c[i] = nn;
                ++nn;
            }
        }
    }
    free(src);
    free(d->bch); free(d->bsum);
    d->nb = nn;
    d->bch = ch;
    d->bsum = (int64_t*)calloc(4 * (size_t)nn, sizeof(int64_t));
    d->bstatw = 0;
    d->bstatw_f = 0.0f;
    d->max_depth_seen = maxd;
}

/* RTSTreeT::Refine (PG.h:1275-1311): the memory-footprint guard, then every leaf whose
 * building stat-weight exceeds the threshold splits; SubDivide (PG.h:1231-1247) gives both
 * children a copy of the DTree wrapper and half the stat-weight, so the split cascades into a
 * complete subtree of depth k = number of halvings while w > th.  Then every leaf runs
 * RTDTreeWrapperT::Reset(maxDepth, subdivTh) (PG.h:1091-1094, RTSTreeWrapperT::Reset
 * PG.h:1650-1655).  The footprint counts 24-byte DTree nodes and 24-byte DTree headers for
 * the building and sampling tree of every STree node, as GetApproxMemoryFootPrint does
 * (PG.h:970-972,1052-1054); interior nodes hold default one-node trees. */
void or_sdtree_refine(void* h, uint64_t spatial_th, int max_mb) {
    OSDTree* t = (OSDTree*)h;
    int do_spatial = 1;
    if (max_mb >= 0) {
        uint64_t fp = 0;
        for (uint32_t i = 0; i < t->nst; ++i) {
            if (t->st[i].child0 >= 0) fp += 96;
            else { const ODTree* d = &t->dt[t->st[i].dtree]; fp += 24ull * (d->nb + d->ns) + 48; }
        }
        if (fp / 1000000 >= (uint64_t)max_mb) do_spatial = 0;
    }
    const float thf = (float)spatial_th;
    if (do_spatial) {
        /* pre-order walk with an explicit stack so that new children are visited too */
        uint32_t cap = 64, top = 0;
        uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        stack[top++] = 0;
        while (top) {
            uint32_t n = stack[--top];
            if (t->st[n].child0 < 0) {
                ODTree* d = &t->dt[t->st[n].dtree];
                if (d->bstatw_f > thf) {
                    const uint32_t c = add_snodes(t, 2);
                    const int32_t dold = t->st[n].dtree;
                    const uint32_t dnew = add_dtree(t);
                    d = &t->dt[dold];
                    ODTree* e = &t->dt[dnew];
                    *e = *d;
                    e->bch = (OChild*)malloc(sizeof(OChild) * d->nb); memcpy(e->bch, d->bch, sizeof(OChild) * d->nb);
                    e->bsum = (int64_t*)malloc(sizeof(int64_t) * 4 * d->nb); memcpy(e->bsum, d->bsum, sizeof(int64_t) * 4 * d->nb);
                    e->sch = (OChild*)malloc(sizeof(OChild) * d->ns); memcpy(e->sch, d->sch, sizeof(OChild) * d->ns);
                    e->ssum = (float*)malloc(sizeof(float) * 4 * d->ns); memcpy(e->ssum, d->ssum, sizeof(float) * 4 * d->ns);
                    d->bstatw_f = d->bstatw_f / 2.0f;
                    e->bstatw_f = d->bstatw_f;
                    t->st[n].child0 = (int32_t)c;
                    t->st[n].dtree = -1;
                    t->st[c].child0 = -1; t->st[c].dtree = dold;
                    t->st[c + 1].child0 = -1; t->st[c + 1].dtree = (int32_t)dnew;
                }
            }
            if (t->st[n].child0 >= 0) {
                if (top + 2 > cap) { cap *= 2; stack = (uint32_t*)realloc(stack, sizeof(uint32_t) * cap); }
                stack[top++] = (uint32_t)t->st[n].child0;
                stack[top++] = (uint32_t)t->st[n].child0 + 1;
            }
        }
        free(stack);
    }
    for (uint32_t i = 0; i < t->ndt; ++i)
        dtree_reset(&t->dt[i], t->max_dtree_depth, t->subdiv_th, t->node_cap, &t->status);
}

/* canonical export, same stream format as the product's rtpg_sdtree_export */
typedef struct { uint8_t* smask; float* scalars; int64_t* counts; uint8_t* dmask; float* dsums;
                 int64_t ns, nl, nd, cs, cl, cd; } OExp;
static void grow(void** p, int64_t* cap, int64_t need, size_t el) {
    if (need <= *cap) return;
    while (*cap < need) *cap = *cap ? 2 * *cap : 1024;
    *p = realloc(*p, (size_t)*cap * el);
}
static void exp_dtree(OExp* e, const OChild* ch, const float* sums_f, const int64_t* sums_i, int bits, uint32_t n) {
    grow((void**)&e->dmask, &e->cd, e->nd + 1, 1);
    int64_t cd4 = e->cd;  /* dsums sized 4 * cd */
    e->dsums = (float*)realloc(e->dsums, (size_t)cd4 * 4 * sizeof(float));
    uint8_t m = 0;
    for (int i = 0; i < 4; ++i) if (ch[n].c[i]) m |= (uint8_t)(1u << i);
    e->dmask[e->nd] = m;
    for (int i = 0; i < 4; ++i) e->dsums[4 * e->nd + i] = sums_f ? sums_f[4 * n + i] : fx_to_float(sums_i[4 * n + i], bits);
    e->nd++;
    for (int i = 0; i < 4; ++i) if (ch[n].c[i]) exp_dtree(e, ch, sums_f, sums_i, bits, ch[n].c[i]);
}
static void exp_stree(OExp* e, const OSDTree* t, uint32_t n, int sampling) {
    grow((void**)&e->smask, &e->cs, e->ns + 1, 1);
    const OSNode s = t->st[n];
    e->smask[e->ns++] = s.child0 >= 0 ? 1 : 0;
    if (s.child0 < 0) {
        const ODTree* d = &t->dt[s.dtree];
        grow((void**)&e->counts, &e->cl, e->nl + 1, sizeof(int64_t));
        e->scalars = (float*)realloc(e->scalars, (size_t)e->cl * 4 * sizeof(float));
        e->scalars[4 * e->nl + 0] = fx_to_float(d->bstatw, t->frac_bits);
        e->scalars[4 * e->nl + 1] = d->s_sum;
        e->scalars[4 * e->nl + 2] = d->s_area;
        e->scalars[4 * e->nl + 3] = d->s_statw;
        const int64_t before = e->nd;
        if (sampling) exp_dtree(e, d->sch, d->ssum, NULL, t->frac_bits, 0);
        else exp_dtree(e, d->bch, NULL, d->bsum, t->frac_bits, 0);
        e->counts[e->nl++] = e->nd - before;
        return;
    }
    exp_stree(e, t, (uint32_t)s.child0, sampling);
    exp_stree(e, t, (uint32_t)s.child0 + 1, sampling);
}
static OExp g_exp;
void or_sdtree_export(void* h, int sampling, int64_t* sizes) {
    free(g_exp.smask); free(g_exp.scalars); free(g_exp.counts); free(g_exp.dmask); free(g_exp.dsums);
    memset(&g_exp, 0, sizeof(g_exp));
    exp_stree(&g_exp, (OSDTree*)h, 0, sampling);
    sizes[0] = g_exp.ns; sizes[1] = g_exp.nl; sizes[2] = g_exp.nd;
}
void or_sdtree_export_copy(uint8_t* smask, float* scalars, int64_t* counts, uint8_t* dmask, float* dsums) {
    memcpy(smask, g_exp.smask, (size_t)g_exp.ns);
    memcpy(scalars, g_exp.scalars, (size_t)g_exp.nl * 4 * sizeof(float));
    memcpy(counts, g_exp.counts, (size_t)g_exp.nl * sizeof(int64_t));
    memcpy(dmask, g_exp.dmask, (size_t)g_exp.nd);
    memcpy(dsums, g_exp.dsums, (size_t)g_exp.nd * 4 * sizeof(float));
}

/* DTreeT::GetMean (PG.h:447-451) */
static inline float dtree_mean(const ODTree* d) {
    if (d->s_statw <= 0.0f) return 0.0f;
    const float factor = O_INV_2PI / (2.0f * d->s_statw);
    return factor * d->s_sum;
}
/* DTreeNodeT::Sample (PG.h:229-277) + DTreeT::Sample (PG.h:478-484) */
static void dtree_sample(const ODTree* d, uint32_t* rng, float* out) {
    if (dtree_mean(d) <= 0.0f) { out[0] = rnd1(rng); out[1] = rnd1(rng); return; }
    uint32_t cur = 0;
    float rx = 0.0f, ry = 0.0f, size = 1.0f;
    for (;;) {
        const float* s = d->ssum + 4 * cur;
        int idx = 0;
        float topLeft = s[0], topRight = s[1];
        float partial = s[0] + s[2];
        float total = s[0] + s[1] + s[2] + s[3];
        float boundary = partial / total;
        float ox = 0.0f, oy = 0.0f;
        float sample = rnd1(rng);
        if (sample < boundary) { sample = sample / boundary; boundary = topLeft / partial; }
        else {
            partial = total - partial; ox = 0.5f;
            sample = (sample - boundary) / (1.0f - boundary);
            boundary = topRight / partial; idx |= 1;
        }
        if (sample >= boundary) { oy = 0.5f; idx |= 2; }
        rx += size * ox; ry += size * oy;
        size *= 0.5f;
        if (d->sch[cur].c[idx] == 0 || s[idx] <= 0.0f) {
            const float a = rnd1(rng), b = rnd1(rng);
            rx += size * a; ry += size * b;
            break;
        }
        cur = d->sch[cur].c[idx];
    }
    out[0] = rx < 0.0f ? 0.0f : (rx > 1.0f ? 1.0f : rx);
    out[1] = ry < 0.0f ? 0.0f : (ry > 1.0f ? 1.0f : ry);
}
/* DTreeNodeT::Pdf (PG.h:279-320) + DTreeT::Pdf (PG.h:485-490) */
static float dtree_pdf(const ODTree* d, float u, float v) {
    if (dtree_mean(d) <= 0.0f) return 1.0f * O_INV_2PI / 2.0f;
    float p[2] = {u, v};
    float result = 1.0f;
    uint32_t cur = 0;
    int idx = quad_child(p);
    for (;;) {
        const float* s = d->ssum + 4 * cur;
        float total = s[0] + s[1] + s[2] + s[3];
        if (s[idx] <= 0.0f) { result = 0.0f; break; }
        const float factor = 4.0f * s[idx] / total;
        result *= factor;
        if (d->sch[cur].c[idx] == 0) break;
        cur = d->sch[cur].c[idx];
        idx = quad_child(p);
    }
    return result * O_INV_2PI / 2.0f;
}
/* guided sample + pdf as SimpleGuide.cu:359-369 uses them */
void or_sdtree_sample_pdf(void* h, int64_t n, const float* pos, const uint32_t* seeds, float* out_uv,
                          float* out_pdf_uv, float* out_dir, float* out_pdf_dir) {
    OSDTree* t = (OSDTree*)h;
    for (int64_t i = 0; i < n; ++i) {
        const ODTree* d = &t->dt[leaf_dtree(t, pos + 3 * i)];
        uint32_t rng = seeds[i];
        float uv[2];
        dtree_sample(d, &rng, uv);
        if (out_uv) { out_uv[2 * i] = uv[0]; out_uv[2 * i + 1] = uv[1]; }
        if (out_pdf_uv) out_pdf_uv[i] = dtree_pdf(d, uv[0], uv[1]);
        if (out_dir || out_pdf_dir) {
            float dir[3];
            canonical_to_dir(uv[0], uv[1], dir);
            normalize3(dir);
            if (out_dir) { out_dir[3 * i] = dir[0]; out_dir[3 * i + 1] = dir[1]; out_dir[3 * i + 2] = dir[2]; }
            if (out_pdf_dir) {
                float c[2];
                or_dir_to_canonical(1, dir, c);
                out_pdf_dir[i] = dtree_pdf(d, c[0], c[1]);
            }
        }
    }
}
void or_sdtree_pdf(void* h, int64_t n, const float* pos, const float* uv, float* out) {
    OSDTree* t = (OSDTree*)h;
    for (int64_t i = 0; i < n; ++i) out[i] = dtree_pdf(&t->dt[leaf_dtree(t, pos + 3 * i)], uv[2 * i], uv[2 * i + 1]);
}
uint32_t or_sdtree_num_stree_nodes(void* h) { return ((OSDTree*)h)->nst; }
uint32_t or_sdtree_num_dtrees(void* h) { return ((OSDTree*)h)->ndt; }

/* Thread-private record target of a tree, for rendering one frame on several host threads
 * into one shared tree: the shadow shares the tree's topology and sampling trees (read only
 * while it exists) and has its own zeroed building sums and stat-weights, which
 * or_sdtree_shadow_merge adds into the tree.  Fixed-point sums make the merged result the
 * same as recording every vertex into the tree on one thread, in any order. */
void* or_sdtree_shadow_new(void* h) {
    const OSDTree* t = (const OSDTree*)h;
    OSDTree* s = (OSDTree*)malloc(sizeof(OSDTree));
    *s = *t;
    s->status = 0;
    s->dt = (ODTree*)malloc(sizeof(ODTree) * (t->ndt ? t->ndt : 1));
    s->capdt = t->ndt;
    for (uint32_t i = 0; i < t->ndt; ++i) {
        s->dt[i] = t->dt[i];
        s->dt[i].bsum = (int64_t*)calloc(4 * (size_t)t->dt[i].nb, sizeof(int64_t));
        s->dt[i].bstatw = 0;
    }
    return s;
}
void or_sdtree_shadow_merge(void* h, void* shadow) {
    OSDTree* t = (OSDTree*)h;
    OSDTree* s = (OSDTree*)shadow;
    for (uint32_t i = 0; i < t->ndt; ++i) {
        for (size_t k = 0; k < 4 * (size_t)t->dt[i].nb; ++k) t->dt[i].bsum[k] += s->dt[i].bsum[k];
        t->dt[i].bstatw += s->dt[i].bstatw;
        free(s->dt[i].bsum);
    }
    t->status |= s->status;
    free(s->dt);
    free(s);
}

/* ------------------------------------------------------------------ hash grid */
/* Cell coordinates as DoubleBufferedHashGrid3T::FindFromCur/Prv compute them
 * (OPX7UtilsGrid.h:189-199): uint(bounds * (p - off) / size), clamped to bounds-1; negative
 * products clamp to 0 (the device conversion semantics). */
static void grid_cell(const float* p, const float* off, const float* size, const uint32_t* b, uint32_t* ijk) {
    for (int k = 0; k < 3; ++k) {
        float f = (p[k] - off[k]) / size[k];
        float s = (float)b[k] * f;
        uint32_t v = s <= 0.0f ? 0u : (s >= 4294967040.0f ? 0xFFFFFFFFu : (uint32_t)s);
        ijk[k] = v > b[k] - 1 ? b[k] - 1 : v;
    }
}
/* DoubleBufferedHashGrid3T::Hash1 / GetCurCellIndex / GetPrvCellIndex (OPX7UtilsGrid.h:241-300) */
void or_hashgrid_insert(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* b,
                        uint32_t nslots, uint32_t* cur, uint32_t* out_slot) {
    const uint32_t nb = nslots / 32;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        grid_cell(pos + 3 * i, off, size, b, c);
        const uint32_t bucket = or_pcg1d(nslots + c[2] + or_pcg1d(c[1] + or_pcg1d(c[0]))) % nb;
        const uint32_t cs = 1u + b[0] * b[1] * c[2] + b[0] * c[1] + c[0];
        uint32_t r = UINT32_MAX;
        for (uint32_t k = 0; k < 32; ++k) {
            uint32_t* s = &cur[32 * bucket + k];
            if (*s == 0) { *s = cs; r = 32 * bucket + k; break; }
            if (*s == cs) { r = 32 * bucket + k; break; }
        }
        out_slot[i] = r;
    }
}
void or_hashgrid_lookup(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* b,
                        uint32_t nslots, const uint32_t* prv, uint32_t* out_slot) {
    const uint32_t nb = nslots / 32;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        grid_cell(pos + 3 * i, off, size, b, c);
        const uint32_t bucket = or_pcg1d(nslots + c[2] + or_pcg1d(c[1] + or_pcg1d(c[0]))) % nb;
        const uint32_t cs = 1u + b[0] * b[1] * c[2] + b[0] * c[1] + c[0];
        uint32_t r = UINT32_MAX;
        for (uint32_t k = 0; k < 32; ++k) {
            const uint32_t s = prv[32 * bucket + k];
            if (s == 0) break;
            if (s == cs) { r = 32 * bucket + k; break; }
        }
        out_slot[i] = r;
    }
}
/* Morton keying (this library's own mode): 21 bits per axis interleaved into 63 bits,
 * key = morton + 1 so that 0 marks an empty slot; bucket = 64-bit mix of the key. */
static uint64_t part1by2_21(uint64_t x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
uint64_t or_morton3(uint32_t x, uint32_t y, uint32_t z) { return part1by2_21(x) | (part1by2_21(y) << 1) | (part1by2_21(z) << 2); }
static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
void or_mhash_insert(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* b,
                     uint32_t nslots, uint64_t* cur, uint32_t* out_slot, uint64_t* out_key) {
    const uint32_t nb = nslots / 32;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        grid_cell(pos + 3 * i, off, size, b, c);
        const uint64_t key = or_morton3(c[0], c[1], c[2]) + 1ull;
        const uint32_t bucket = (uint32_t)(mix64(key) % nb);
        uint32_t r = UINT32_MAX;
        for (uint32_t k = 0; k < 32; ++k) {
            uint64_t* s = &cur[32 * (uint64_t)bucket + k];
            if (*s == 0) { *s = key; r = 32 * bucket + k; break; }
            if (*s == key) { r = 32 * bucket + k; break; }
        }
        out_slot[i] = r;
        if (out_key) out_key[i] = key;
    }
}
void or_mhash_lookup(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* b,
                     uint32_t nslots, const uint64_t* prv, uint32_t* out_slot) {
    const uint32_t nb = nslots / 32;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        grid_cell(pos + 3 * i, off, size, b, c);
        const uint64_t key = or_morton3(c[0], c[1], c[2]) + 1ull;
        const uint32_t bucket = (uint32_t)(mix64(key) % nb);
        uint32_t r = UINT32_MAX;
        for (uint32_t k = 0; k < 32; ++k) {
            const uint64_t s = prv[32 * (uint64_t)bucket + k];
            if (s == 0) break;
            if (s == key) { r = 32 * bucket + k; break; }
        }
        out_slot[i] = r;
    }
}

/* ------------------------------------------------------------------ Morton quadtree */
/* MortonUtils::Part1By1_16 (OPX7UtilsMorton.h:41-64); code = (part(y) << 1) + part(x)
 * (Morton2Utils::GetCodeFromPosIdx, :165-167). */
static uint32_t part1by1(uint32_t x) {
    x &= 0x0000FFFF;
    x = (x ^ (x << 8)) & 0x00FF00FF;
    x = (x ^ (x << 4)) & 0x0F0F0F0F;
    x = (x ^ (x << 2)) & 0x33333333;
    x = (x ^ (x << 1)) & 0x55555555;
    return x;
}
static uint32_t compact1by1(uint32_t x) {
    x &= 0x55555555;
    x = (x ^ (x >> 1)) & 0x33333333;
    x = (x ^ (x >> 2)) & 0x0F0F0F0F;
    x = (x ^ (x >> 4)) & 0x00FF00FF;
    x = (x ^ (x >> 8)) & 0x0000FFFF;
    return x;
}
uint32_t or_morton2(uint32_t x, uint32_t y) { return (part1by1(y) << 1) + part1by1(x); }
static inline uint32_t mqt_off(uint32_t level) { return ((1u << (2 * level)) - 1u) / 3u; }
/* MortonQuadTreeT::Record (OPX7UtilsMorton.h:262-285, leaf only): pos = uint(uv * 2^L),
 * clamped to 2^L - 1 (uv == 1 would address past the level).  Leaves accumulate in fixed
 * point: leaves[cell * 4^L + code]. */
void or_mqt_record(int64_t n, uint32_t level, int bits, int64_t* leaves, const uint32_t* cell, const float* uv,
                   const float* value, uint32_t* status) {
    const float numNodes = ldexpf(1.0f, (int)level);
    const uint32_t maxi = (1u << level) - 1u;
    for (int64_t i = 0; i < n; ++i) {
        if (cell[i] == UINT32_MAX) continue;
        const float v = value[i];
        if (!(isfinite(v) && v > 0.0f)) continue;
        uint32_t px = (uint32_t)(uv[2 * i] * numNodes), py = (uint32_t)(uv[2 * i + 1] * numNodes);
        px = px > maxi ? maxi : px;
        py = py > maxi ? maxi : py;
        leaves[((uint64_t)cell[i] << (2 * level)) + or_morton2(px, py)] += to_fx(v, bits, status);
    }
}
/* mortonBuildKernel (OPX7UtilsMortonBuild.cu:2-16): the pyramid of a cell; here from exact
 * integer leaf sums, each level converted to float once. */
void or_mqt_build(uint32_t ncells, uint32_t level, int bits, const int64_t* leaves, float* pyramid) {
    const uint32_t per = mqt_off(level + 1), nl = 1u << (2 * level);
    int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * per);
    for (uint32_t c = 0; c < ncells; ++c) {
        const int64_t* lf = leaves + (uint64_t)c * nl;
        memcpy(tmp + mqt_off(level), lf, sizeof(int64_t) * nl);
        for (int l = (int)level - 1; l >= 0; --l) {
            const uint32_t o = mqt_off((uint32_t)l), oc = mqt_off((uint32_t)l + 1), cnt = 1u << (2 * l);
            for (uint32_t k = 0; k < cnt; ++k)
                tmp[o + k] = tmp[oc + 4 * k] + tmp[oc + 4 * k + 1] + tmp[oc + 4 * k + 2] + tmp[oc + 4 * k + 3];
        }
        float* w = pyramid + (uint64_t)c * per;
        for (uint32_t k = 0; k < per; ++k) w[k] = fx_to_float(tmp[k], bits);
    }
    free(tmp);
}
/* MortonQuadTreeT::SampleAndPdf (OPX7UtilsMorton.h:286-344) for one pyramid w; an empty tree
 * samples uniformly with pdf 1. */
static void mqt_sample_one(const float* w, uint32_t level, uint32_t* rng, float* ux, float* uy, float* pdf) {
    float total = w[0];
    if (total <= 0.0f) {
        *ux = rnd1(rng); *uy = rnd1(rng); *pdf = 1.0f;
        return;
    }
    uint32_t size = 4, offset = 1, code = 0;
    for (uint32_t l = 0; l < level; ++l) {
        const float* q = w + offset + (code << 2);
        uint32_t cl = 0;
        float partial = q[0] + q[2];
        float boundary = partial / total;
        float sample = rnd1(rng);
        if (sample < boundary) { sample /= boundary; boundary = q[0] / partial; }
        else {
            partial = q[1] + q[3];
            sample = (sample - boundary) / (1.0f - boundary);
            boundary = q[1] / partial;
            cl |= 1;
        }
        if (sample >= boundary) cl |= 2;
        total = q[cl];
        code = (code << 2) + cl;
        offset += size;
        size *= 4;
    }
    const float nn = ldexpf(1.0f, (int)level);
    const uint32_t xi = compact1by1(code), yi = compact1by1(code >> 1);
    *ux = ((float)xi + rnd1(rng)) / nn;
    *uy = ((float)yi + rnd1(rng)) / nn;
    *pdf = total / w[0] * ldexpf(1.0f, (int)(2 * level));
}
/* MortonQuadTreeT::Pdf (OPX7UtilsMorton.h:401-414); an empty tree has pdf 1 */
static float mqt_pdf_one(const float* w, uint32_t level, float u, float v) {
    if (w[0] <= 0.0f) return 1.0f;
    const float nn = ldexpf(1.0f, (int)level);
    const uint32_t maxi = (1u << level) - 1u;
    uint32_t px = (uint32_t)(u * nn), py = (uint32_t)(v * nn);
    px = px > maxi ? maxi : px;
    py = py > maxi ? maxi : py;
    return w[mqt_off(level) + or_morton2(px, py)] / w[0] * nn * nn;
}
void or_mqt_sample_pdf(int64_t n, uint32_t level, const float* pyramid, const uint32_t* cell, const uint32_t* seeds,
                       float* out_uv, float* out_pdf, float* out_pdf_eval) {
    const uint32_t per = mqt_off(level + 1);
    for (int64_t i = 0; i < n; ++i) {
        const float* w = pyramid + (uint64_t)cell[i] * per;
        uint32_t rng = seeds[i];
        float ux, uy, pdf;
        mqt_sample_one(w, level, &rng, &ux, &uy, &pdf);
        out_uv[2 * i] = ux; out_uv[2 * i + 1] = uy;
        out_pdf[i] = pdf;
        if (out_pdf_eval) out_pdf_eval[i] = mqt_pdf_one(w, level, ux, uy);
    }
}

/* ------------------------------------------------------------------ integrator
 * CPU restatement of RTLib's guided path tracer for small scenes (brute-force intersection):
 *   raygen       SimpleGuide.cu:48-156 (jitter, bounce loop, trace vertices, commit)
 *   closest hit  SimpleGuide.cu:287-520 (Phong/Lambert BSDF, guide mixture, NEE, RIS, glass,
 *                emission rule), miss SimpleGuide.cu:202-219
 *   lights       MeshLightList::Sample / MeshLight::Sample (SimpleKernel.h:81-122)
 *   reservoir    Reservoir::Update (SimpleKernel.h:124-143)
 *   commit       TraceVertexT::Commit (OPX7UtilsPathGuiding.h:830-866)
 * The random numbers are drawn in the order the device code draws them (argument lists
 * evaluated left to right), so a CPU path and a GPU path with the same seed follow the same
 * decisions until float differences in transcendental functions separate them. */
typedef struct { float x, y, z; } V3;
static inline V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 vs(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
static inline V3 vdivs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float vlen(V3 a) { return sqrtf(vdot(a, a)); }
static inline V3 vunit(V3 a) { return vdivs(a, vlen(a)); }
static inline float vavg(V3 a) { return (a.x + a.y + a.z) / 3.0f; }
static inline int vnan(V3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
static inline float sinpi_f(float x) { return (float)sin(3.14159265358979323846 * (double)x); }
static inline float cospi_f(float x) { return (float)cos(3.14159265358979323846 * (double)x); }

typedef struct {
    float diffuse[3]; int32_t tex; float specular[3]; float shininess; float emission[3]; float ref_index;
    int32_t type; int32_t pad[3];
} OMat;
typedef struct {
    const float* tri_v; const uint32_t* tri_mat; const float* tri_uv; uint32_t ntris;
    const OMat* mats; const uint32_t* light_tris; const uint32_t* light_first; const uint32_t* light_count;
    const float* light_emit; uint32_t nlights;
    const float* tex; uint32_t tex_w, tex_h;
    float eye[3], cu[3], cv[3], cw[3], bg[3];
    uint32_t width, height, max_depth, num_candidates;
    float fraction; /* guide/BSDF mixing fraction of the SD-tree (STreeT::fraction) */
    const float* tri_xf; /* 12 floats per triangle: the rows of or_tri_transforms */
} OScene;

static V3 tri_vert(const OScene* s, uint32_t t, int k) {
    const float* p = s->tri_v + 9 * (size_t)t + 3 * k;
    return v3(p[0], p[1], p[2]);
}
/* The rows of the world -> triangle-frame map of every triangle (Baldwin and Weber, "Fast
 * Ray-Triangle Intersections by Coordinate Transformation", JCGT 5(3), 2016), as the device's
 * tri_transform forms them: with e1 = v1 - v0, e2 = v2 - v0, n = e1 x e2, the rows of the
 * inverse of [e1 e2 n] are (e2 x n, n x e1, n) / |n|^2, translated by -v0; all in double
 * (rounded as written), then rounded to float.  Row 0 gives u, row 1 v, row 2 the offset along
 * the normal. */
void or_tri_transforms(const float* tri_v, uint32_t n, float* out) {
    for (uint32_t t = 0; t < n; ++t) {
        const float* v = tri_v + 9 * (size_t)t;
        const double ax = v[0], ay = v[1], az = v[2];
        const double e1x = (double)v[3] - ax, e1y = (double)v[4] - ay, e1z = (double)v[5] - az;
        const double e2x = (double)v[6] - ax, e2y = (double)v[7] - ay, e2z = (double)v[8] - az;
        const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
        const double nn = nx * nx + ny * ny + nz * nz;
        const double m[3][3] = {{e2y * nz - e2z * ny, e2z * nx - e2x * nz, e2x * ny - e2y * nx},
                                {ny * e1z - nz * e1y, nz * e1x - nx * e1z, nx * e1y - ny * e1x},
                                {nx, ny, nz}};
        float* r = out + 12 * (size_t)t;
        for (int k = 0; k < 3; ++k) {
            const double w = -(m[k][0] * ax + m[k][1] * ay + m[k][2] * az);
            r[4 * k] = (float)(m[k][0] / nn);
            r[4 * k + 1] = (float)(m[k][1] / nn);
            r[4 * k + 2] = (float)(m[k][2] / nn);
            r[4 * k + 3] = (float)(w / nn);
        }
    }
}
/* row . d (no offset) and row . o + offset, as chains of fused multiply-adds */
static float xf_dir(const float* r, V3 d) { return fmaf(r[0], d.x, fmaf(r[1], d.y, r[2] * d.z)); }
static float xf_pt(const float* r, V3 o) { return fmaf(r[0], o.x, fmaf(r[1], o.y, fmaf(r[2], o.z, r[3]))); }
/* Closest (any = 0) or any (any = 1) hit in (tmin, tmax) over every triangle in scene order,
 * the device's tri_hit: t = -(r2 . o + w2) / (r2 . d) with the correctly rounded reciprocal,
 * u and v as the point's coordinates plus t times the direction's; the lowest index wins a tie. */
static int o_trace(const OScene* s, V3 o, V3 d, float tmin, float tmax, int any, float* th, uint32_t* prim, float* hu,
                   float* hv) {
    int hit = 0;
    float best = tmax;
    for (uint32_t t = 0; t < s->ntris; ++t) {
        const float* r = s->tri_xf + 12 * (size_t)t;
        const float den = xf_dir(r + 8, d), num = xf_pt(r + 8, o);
        const float tt = -num * (1.0f / den);
        const float u = fmaf(tt, xf_dir(r, d), xf_pt(r, o));
        const float v = fmaf(tt, xf_dir(r + 4, d), xf_pt(r + 4, o));
        if (tt > tmin && tt < best && u >= 0.0f && v >= 0.0f && u + v <= 1.0f) {
            best = tt; hit = 1;
            if (th) *th = tt;
            if (prim) *prim = t;
            if (hu) *hu = u;
            if (hv) *hv = v;
            if (any) return 1;
        }
    }
    return hit;
}
/* Batched o_trace over a triangle list (the brute-force check of the device hit queries). */
void or_intersect(const float* tri_v, uint32_t ntris, int64_t n, const float* org, const float* dir, float tmin,
                  float tmax, int any, float* out_t, uint32_t* out_prim) {
    OScene s;
    memset(&s, 0, sizeof(s));
    float* xf = (float*)malloc(12 * sizeof(float) * (ntris ? ntris : 1));
    or_tri_transforms(tri_v, ntris, xf);
    s.tri_v = tri_v;
    s.ntris = ntris;
    s.tri_xf = xf;
    for (int64_t i = 0; i < n; ++i) {
        float t = -1.0f;
        uint32_t p = 0xffffffffu;
        V3 o = v3(org[3 * i], org[3 * i + 1], org[3 * i + 2]), d = v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        if (!o_trace(&s, o, d, tmin, tmax, any, &t, &p, 0, 0)) { t = -1.0f; p = 0xffffffffu; }
        out_t[i] = t;
        out_prim[i] = p;
    }
    free(xf);
}
typedef struct { V3 t, b, n; } OOnb;
static OOnb onb(V3 normal) {
    OOnb r;
    r.n = vunit(normal);
    if (fabsf(r.n.x) > fabsf(r.n.z)) r.b = v3(-r.n.y, r.n.x, 0.0f);
    else r.b = v3(0.0f, -r.n.z, r.n.y);
    r.b = vunit(r.b);
    r.t = vunit(vcross(r.n, r.b));
    return r;
}
static V3 onb_local(OOnb o, V3 d) { return vadd(vadd(vs(d.x, o.t), vs(d.y, o.b)), vs(d.z, o.n)); }
/* sampleCosinePDF (SimpleGuide.cu:28-33): ONB(normal).local(random_cosine_direction(rng))
 * (VectorFunction.h:5666-5697, Random.h:321-334); sin / cos of 2 pi x as sinpi / cospi of 2x */
static V3 o_sample_cosine(V3 normal, uint32_t* rng) {
    float a = rnd1(rng), c = rnd1(rng);
    float r = sqrtf(a), z = sqrtf(1.0f - a);
    return onb_local(onb(normal), v3(r * cospi_f(2.0f * c), r * sinpi_f(2.0f * c), z));
}
/* samplePhongPDF (SimpleGuide.cu:34-42): cos theta = u^(1/(s+1)), phi = 2 pi u' around refl */
static V3 o_sample_phong(V3 refl, float shininess, uint32_t* rng) {
    float cosT = powf(rnd1(rng), 1.0f / (shininess + 1.0f));
    float sinT = sqrtf(fmaxf(1.0f - cosT * cosT, 0.0f));
    float phi = O_2PI * rnd1(rng);
    return onb_local(onb(refl), v3(sinT * cosf(phi), sinT * sinf(phi), cosT));
}
static float phong_pdf_o(V3 d, V3 refl, float s) {
    float c = vdot(refl, d);
    c = c > 0.0f ? c : 0.0f;
    return (s + 1.0f) * powf(c, s) * O_INV_2PI;
}
static V3 reflect_o(V3 d, V3 n) { return vsub(d, vs(2.0f * vdot(d, n), n)); }
static V3 phong_bsdf_o(V3 kd, V3 ks, float s, V3 d, V3 refl) {
    return vadd(vs((float)0.318309886183790691216444201927515678107738494873046875, kd),
                vs(phong_pdf_o(d, refl, s), vs((s + 2.0f) / (s + 1.0f), ks)));
}
typedef struct { V3 dir, normal, emission, pos; float dist, inv_pdf; } OLight;
/* random_in_unit_triangle (Random.h:289-296): a = min, b = max of two uniforms,
 * v0 a + v1 (1 - b) + v2 (b - a).  MeshLight::Sample forms the same point through
 * barycentrics of the unit vectors (SimpleKernel.h:81-98), bit for bit the same floats. */
static V3 o_random_in_unit_triangle(V3 v0, V3 v1, V3 v2, uint32_t* rng) {
    float r0 = rnd1(rng), r1 = rnd1(rng);
    float a = fminf(r0, r1), b = fmaxf(r0, r1);
    return vadd(vadd(vs(a, v0), vs(1.0f - b, v1)), vs(b - a, v2));
}
/* Reservoir::Update (SimpleKernel.h:124-143): w_sum += w_i, ++m, keep x_i iff
 * w_i / w_sum >= rnd01.  Returns whether x_i was kept. */
static int o_reservoir_update(float* w_sum, uint32_t* m, float w_i, float rnd01) {
    *w_sum += w_i;
    ++*m;
    return (w_i / *w_sum) >= rnd01;
}
/* MeshLightList::Sample -> MeshLight::Sample (SimpleKernel.h:81-122) with white emission
 * textures: mesh next() % count, triangle next() % indCount, invPdf = area * indCount * count */
static OLight o_sample_light(const OScene* s, V3 p_in, uint32_t* rng) {
    uint32_t mi = xs32_next(rng) % s->nlights;
    uint32_t ti = s->light_tris[s->light_first[mi] + xs32_next(rng) % s->light_count[mi]];
    V3 v0 = tri_vert(s, ti, 0), v1 = tri_vert(s, ti, 1), v2 = tri_vert(s, ti, 2);
    V3 nf = vcross(vsub(v1, v0), vsub(v2, v0));
    V3 p = o_random_in_unit_triangle(v0, v1, v2, rng);
    V3 d = vsub(p, p_in);
    OLight l;
    l.pos = p;
    l.dist = vlen(d);
    l.dir = vunit(d);
    l.emission = v3(s->light_emit[3 * mi], s->light_emit[3 * mi + 1], s->light_emit[3 * mi + 2]);
    l.normal = vunit(nf);
    l.inv_pdf = vlen(nf) / 2.0f * (float)s->light_count[mi] * (float)s->nlights;
    return l;
}
#define O_NEE 1u
#define O_RIS 2u
#define O_GRID 4u
#define O_TREE 8u
#define O_BUILD 16u
#define O_FINAL 32u
#define O_LOCATE 64u
#define O_KTV 10
typedef struct { V3 pos, dir, thr, rad, bsdf; float wopdf, cosine; int valid, delta; uint32_t cell; } OVert;

/* The hash-grid guide of SimpleGuide2.cu: DoubleBufferedHashGrid3T (cur / prv tables of
 * 64-bit keys, 0 = empty) and one Morton quadtree per slot (int64 building leaves, float
 * sampling pyramid).  keying 0: the reference's pcg1d bucket and checksum key; 1: 63-bit
 * Morton key + 1 with a 64-bit mixed bucket. */
typedef struct {
    float off[3], size[3];
    uint32_t bounds[3], nslots;
    int32_t keying;
    uint64_t* cur;
    uint64_t* prv;
    uint32_t level;
    int32_t bits;
    int64_t* leaves;
    const float* pyramid;
    float fraction;
    uint32_t status;
} OGrid;
static uint64_t grid_key(const OGrid* g, V3 p, uint32_t* bucket) {
    float pp[3] = {p.x, p.y, p.z};
    uint32_t c[3];
    grid_cell(pp, g->off, g->size, g->bounds, c);
    const uint32_t nb = g->nslots / 32;
    if (g->keying == 0) {
        *bucket = or_pcg1d(g->nslots + c[2] + or_pcg1d(c[1] + or_pcg1d(c[0]))) % nb;
        return (uint64_t)(1u + g->bounds[0] * g->bounds[1] * c[2] + g->bounds[0] * c[1] + c[0]);
    }
    const uint64_t key = or_morton3(c[0], c[1], c[2]) + 1ull;
    *bucket = (uint32_t)(mix64(key) % nb);
    return key;
}
/* FindFromPrv (OPX7UtilsGrid.h:278-300) */
static uint32_t grid_find_prv(const OGrid* g, uint64_t key, uint32_t b) {
    for (uint32_t k = 0; k < 32; ++k) {
        const uint64_t v = g->prv[32 * (uint64_t)b + k];
        if (v == 0) return UINT32_MAX;
        if (v == key) return 32 * b + k;
    }
    return UINT32_MAX;
}
/* FindFromCur (OPX7UtilsGrid.h:189-226) */
static uint32_t grid_insert_cur(OGrid* g, uint64_t key, uint32_t b) {
    for (uint32_t k = 0; k < 32; ++k) {
        uint64_t* v = &g->cur[32 * (uint64_t)b + k];
        if (*v == 0) { *v = key; return 32 * b + k; }
        if (*v == key) return 32 * b + k;
    }
    g->status |= 0x10u;
    return UINT32_MAX;
}
/* MortonTraceVertexT::Commit (OPX7UtilsMorton.h:550-585) -> MortonQuadTreeWrapperT::Record */
static void commit_vertex_grid(OGrid* g, const OVert* v) {
    if (!v->valid || v->delta) return;
    V3 r = v->rad, b = v->bsdf;
    int okr = isfinite(r.x) && r.x >= 0.f && isfinite(r.y) && r.y >= 0.f && isfinite(r.z) && r.z >= 0.f;
    int okb = isfinite(b.x) && b.x >= 0.f && isfinite(b.y) && b.y >= 0.f && isfinite(b.z) && b.z >= 0.f;
    if (v->wopdf <= 0.0f || !okr || !okb) return;
    V3 lr = v3(0, 0, 0);
    if (v->thr.x * v->wopdf > 1e-4f) lr.x = r.x / v->thr.x;
    if (v->thr.y * v->wopdf > 1e-4f) lr.y = r.y / v->thr.y;
    if (v->thr.z * v->wopdf > 1e-4f) lr.z = r.z / v->thr.z;
    lr = vs(fabsf(v->cosine), lr);
    float lavg = (lr.x + lr.y + lr.z) / 3.0f;
    float irr = lavg / v->wopdf;
    float d[3] = {v->dir.x, v->dir.y, v->dir.z}, uv[2];
    or_dir_to_canonical(1, d, uv);
    or_mqt_record(1, g->level, g->bits, g->leaves, &v->cell, uv, &irr, &g->status);
}

static void commit_vertex(OSDTree* t, const OVert* v) {
    if (!v->valid || v->delta) return;
    V3 r = v->rad, b = v->bsdf;
    int okr = isfinite(r.x) && r.x >= 0.f && isfinite(r.y) && r.y >= 0.f && isfinite(r.z) && r.z >= 0.f;
    int okb = isfinite(b.x) && b.x >= 0.f && isfinite(b.y) && b.y >= 0.f && isfinite(b.z) && b.z >= 0.f;
    if (v->wopdf <= 0.0f || !okr || !okb) return;
    V3 lr = v3(0, 0, 0);
    if (v->thr.x * v->wopdf > 1e-4f) lr.x = r.x / v->thr.x;
    if (v->thr.y * v->wopdf > 1e-4f) lr.y = r.y / v->thr.y;
    if (v->thr.z * v->wopdf > 1e-4f) lr.z = r.z / v->thr.z;
    lr = vs(fabsf(v->cosine), lr);
    float lavg = (lr.x + lr.y + lr.z) / 3.0f;
    float pos[3] = {v->pos.x, v->pos.y, v->pos.z}, d[3] = {v->dir.x, v->dir.y, v->dir.z}, uv[2];
    or_dir_to_canonical(1, d, uv);
    float one = 1.0f;
    or_sdtree_record(t, 1, pos, uv, &lavg, &v->wopdf, &one, NULL);
}

/* The closest-hit shading of one path vertex, as RTLib's __closesthit__radiance does it
 * (SimpleGuide.cu:287-497; the hash-grid guide of SimpleGuide2.cu:285-523): BSDF / guide
 * mixture sampling, NEE or RIS with its shadow ray, the glass branch, the emission rule.
 * In: the ray (org, dir), its hit (t, prim, barycentrics hu, hv), the throughput, hit flags
 * and depth of the path before the vertex, its Xorshift32 state.  Out: the next ray, the
 * throughput after the vertex (zero unless a Phong or glass branch sets it, as
 * currThroughput starts), the radiance the vertex adds (L), its hit flags and, for the grid
 * guide, its cell. */
typedef struct {
    V3 position, direction, cur_thr, bsdf_val, L;
    float cosine, wo_pdf;
    uint32_t hflags, cell;
} OShade;
static void o_shade(const OScene* s, uint32_t flags, OSDTree* tree, OGrid* grid, V3 org, V3 dir, float t,
                    uint32_t prim, float hu, float hv, V3 thr, uint32_t pflags, uint32_t depth, uint32_t* prng,
                    OShade* out) {
    const int use_tree = (flags & O_TREE) != 0, use_grid = (flags & O_GRID) != 0, build = (flags & O_BUILD) != 0;
    const uint32_t mqt_per = use_grid ? mqt_off(grid->level + 1) : 0;
    const float inv_pi = (float)0.318309886183790691216444201927515678107738494873046875;
    uint32_t rng = *prng;
    V3 L = v3(0, 0, 0), cur_thr = v3(0, 0, 0), direction = v3(0, 0, 0), bsdf_val = v3(0, 0, 0);
    float cosine = 0.0f, wo_pdf = 0.0f;
    uint32_t hflags = 0;
    V3 position = org;
    V3 v0 = tri_vert(s, prim, 0), v1 = tri_vert(s, prim, 1), v2 = tri_vert(s, prim, 2);
    V3 fn = vunit(vcross(vsub(v1, v0), vsub(v2, v0)));
    position = vadd(org, vs(t, dir));
    const OMat* m = &s->mats[s->tri_mat[prim]];
    V3 diffuse = v3(m->diffuse[0], m->diffuse[1], m->diffuse[2]);
    V3 spec = v3(m->specular[0], m->specular[1], m->specular[2]);
    V3 emis = v3(m->emission[0], m->emission[1], m->emission[2]);
    if (m->tex >= 0 && s->tex && s->tri_uv) {
        const float* uv = s->tri_uv + 6 * (size_t)prim;
        float w0 = 1.0f - hu - hv;
        float tu = w0 * uv[0] + hu * uv[2] + hv * uv[4], tv = w0 * uv[1] + hu * uv[3] + hv * uv[5];
        float fu = tu - floorf(tu), fv = tv - floorf(tv);
        uint32_t ix = (uint32_t)(fu * s->tex_w), iy = (uint32_t)(fv * s->tex_h);
        if (ix > s->tex_w - 1) ix = s->tex_w - 1;
        if (iy > s->tex_h - 1) iy = s->tex_h - 1;
        const float* px = s->tex + 3 * ((size_t)iy * s->tex_w + ix);
        diffuse = vmul(diffuse, v3(px[0], px[1], px[2]));
    }
    int count_emitted = (pflags & 8u) || m->type == 3;
    uint32_t dt = 0, cell = UINT32_MAX;
    if (use_tree) dt = (uint32_t)leaf_dtree(tree, &position.x);
    if (m->type == 0) {
        uint32_t gb = 0, prv_cell = UINT32_MAX;
        uint64_t gk = 0;
        if (use_grid) {
            gk = grid_key(grid, position, &gb);
            prv_cell = grid_find_prv(grid, gk, gb);
        }
        V3 refl = vunit(reflect_o(dir, fn));
        V3 d0 = o_sample_cosine(fn, &rng);
        V3 d1 = o_sample_phong(refl, m->shininess, &rng);
        float c0 = vdot(d0, fn), c1 = vdot(d1, fn);
        float cp0 = fmaxf(c0 * inv_pi, 0.0f), cp1 = fmaxf(c1 * inv_pi, 0.0f);
        float pp0 = phong_pdf_o(d0, refl, m->shininess), pp1 = phong_pdf_o(d1, refl, m->shininess);
        float ad = 1.0e-10f + vavg(diffuse), as = 1.0e-10f + vavg(spec);
        float sel = ad / (ad + as);
        float sf = (m->shininess + 2.0f) / (m->shininess + 1.0f);
        float bsdf_pdf;
        if (rnd1(&rng) < sel) {
            direction = d0; cosine = c0;
            bsdf_val = vadd(vs(inv_pi, diffuse), vs(pp0, vs(sf, spec)));
            bsdf_pdf = sel * cp0 + (1.0f - sel) * pp0;
        } else {
            direction = d1; cosine = c1;
            bsdf_val = vadd(vs(inv_pi, diffuse), vs(pp1, vs(sf, spec)));
            bsdf_pdf = sel * cp1 + (1.0f - sel) * pp1;
        }
        if (use_tree && build) {
            const ODTree* dd = &tree->dt[dt];
            if (rnd1(&rng) < s->fraction) {
                float uv[2];
                dtree_sample(dd, &rng, uv);
                float dv[3];
                const float cosTheta = 2.0f * uv[0] - 1.0f;
                const float sinTheta = sqrtf(fmaxf(1.0f - cosTheta * cosTheta, 0.0f));
                dv[0] = sinTheta * cospi_f(2.0f * uv[1]);
                dv[1] = sinTheta * sinpi_f(2.0f * uv[1]);
                dv[2] = cosTheta;
                float l = 1.0f / sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                direction = v3(dv[0] * l, dv[1] * l, dv[2] * l);
                cosine = vdot(direction, fn);
                float cp2 = fmaxf(cosine * inv_pi, 0.0f);
                float pp2 = phong_pdf_o(direction, refl, m->shininess);
                bsdf_val = vadd(vs(inv_pi, diffuse), vs(pp2, vs(sf, spec)));
                bsdf_pdf = sel * cp2 + (1.0f - sel) * pp2;
            }
            float dd3[3] = {direction.x, direction.y, direction.z}, c2[2];
            or_dir_to_canonical(1, dd3, c2);
            float dpdf = fmaxf(dtree_pdf(dd, c2[0], c2[1]), 0.0f);
            wo_pdf = (1.0f - s->fraction) * bsdf_pdf + s->fraction * dpdf;
        } else if (use_grid && build && prv_cell != UINT32_MAX) {
            /* SimpleGuide2.cu:350-377 */
            const float* w = grid->pyramid + (uint64_t)prv_cell * mqt_per;
            float dpdf;
            if (rnd1(&rng) < grid->fraction) {
                float uv[2], tp;
                mqt_sample_one(w, grid->level, &rng, &uv[0], &uv[1], &tp);
                dpdf = (float)((double)tp * (0.25 * 0.318309886183790691216444201927515678107738494873046875));
                float dv[3];
                const float cosTheta = 2.0f * uv[0] - 1.0f;
                const float sinTheta = sqrtf(fmaxf(1.0f - cosTheta * cosTheta, 0.0f));
                dv[0] = sinTheta * cospi_f(2.0f * uv[1]);
                dv[1] = sinTheta * sinpi_f(2.0f * uv[1]);
                dv[2] = cosTheta;
                float l = 1.0f / sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                direction = v3(dv[0] * l, dv[1] * l, dv[2] * l);
                cosine = vdot(direction, fn);
                float cp2 = fmaxf(cosine * inv_pi, 0.0f);
                float pp2 = phong_pdf_o(direction, refl, m->shininess);
                bsdf_val = vadd(vs(inv_pi, diffuse), vs(pp2, vs(sf, spec)));
                bsdf_pdf = sel * cp2 + (1.0f - sel) * pp2;
            } else {
                float dd3[3] = {direction.x, direction.y, direction.z}, c2[2];
                or_dir_to_canonical(1, dd3, c2);
                const float tp = mqt_pdf_one(w, grid->level, c2[0], c2[1]);
                dpdf = fmaxf((float)((double)(tp * 0.25f) * 0.318309886183790691216444201927515678107738494873046875), 0.0f);
            }
            wo_pdf = grid->fraction * dpdf + (1.0f - grid->fraction) * bsdf_pdf;
        } else {
            wo_pdf = bsdf_pdf;
        }
        cur_thr = wo_pdf > 0.0f ? vmul(thr, vdivs(vs(fmaxf(cosine, 0.0f), bsdf_val), wo_pdf)) : v3(0, 0, 0);
        if (flags & O_NEE) {
            if (depth < s->max_depth - 1 && s->nlights > 0) {
                if (flags & O_RIS) {
                    float w_sum = 0.0f, fay = 0.0f, disty = 0.0f;
                    uint32_t mc = 0;
                    V3 fy = v3(0, 0, 0), ldy = v3(0, 0, 0);
                    for (uint32_t k = 0; k < s->num_candidates; ++k) {
                        OLight l = o_sample_light(s, position, &rng);
                        float ndl = vdot(l.dir, fn), lndl = -vdot(l.dir, l.normal);
                        V3 b = phong_bsdf_o(diffuse, spec, m->shininess, l.dir, refl);
                        float g = fmaxf(ndl, 0.0f) * fmaxf(lndl, 0.0f) / (l.dist * l.dist);
                        V3 f = vmul(vmul(b, l.emission), v3(g, g, g));
                        float fa = vavg(f), wi = fa * l.inv_pdf;
                        if (o_reservoir_update(&w_sum, &mc, wi, rnd1(&rng))) { fy = f; fay = fa; ldy = l.dir; disty = l.dist; }
                    }
                    if (w_sum > 0.0f && fay > 0.0f &&
                        !o_trace(s, position, ldy, 0.0001f, disty - 0.0001f, 1, 0, 0, 0, 0))
                        L = vadd(L, vs(w_sum / (fay * (float)mc), vmul(thr, fy)));
                } else {
                    OLight l = o_sample_light(s, position, &rng);
                    V3 b = phong_bsdf_o(diffuse, spec, m->shininess, l.dir, refl);
                    float g = fmaxf(-vdot(l.dir, l.normal), 0.0f) * fabsf(vdot(l.dir, fn)) / (l.dist * l.dist);
                    if (!o_trace(s, position, l.dir, 0.0001f, l.dist - 0.0001f, 1, 0, 0, 0, 0))
                        L = vadd(L, vs(l.inv_pdf, vs(g, vmul(vmul(thr, b), l.emission))));
                }
            }
        } else {
            hflags |= 8u;
        }
        if (use_grid)
            cell = ((flags & O_LOCATE) && prv_cell == UINT32_MAX) ? grid_insert_cur(grid, gk, gb) : prv_cell;
    } else if (m->type == 1) {
        V3 rn;
        float rri, ci = vdot(fn, dir);
        if (ci < 0.0f) { rn = fn; rri = 1.0f / m->ref_index; ci = -ci; }
        else { rn = v3(-fn.x, -fn.y, -fn.z); rri = m->ref_index; }
        float so2 = (1.0f - ci * ci) * (rri * rri);
        float f0 = ((1.0f - rri) / (1.0f + rri)) * ((1.0f - rri) / (1.0f + rri));
        float om = 1.0f - ci;
        float fres = f0 + (1.0f - f0) * (om * om * om * om * om);
        V3 rd = vunit(reflect_o(dir, rn));
        if (rnd1(&rng) < fres || so2 > 1.0f) {
            position = vadd(position, vs(0.0001f, rn));
            direction = rd; cosine = fabsf(ci); bsdf_val = spec; cur_thr = vmul(thr, spec);
        } else {
            position = vsub(position, vs(0.0001f, rn));
            float si2 = fmaxf(1.0f - ci * ci, 0.0f), co = sqrtf(1.0f - so2);
            V3 rf;
            if (si2 > 0.0f) rf = vunit(vsub(vs(sqrtf(so2), vdivs(vadd(dir, vs(ci, rn)), sqrtf(si2))), vs(co, rn)));
            else rf = dir;
            direction = rf; cosine = fabsf(vdot(rf, rn)); bsdf_val = v3(1, 1, 1); cur_thr = thr;
        }
        wo_pdf = fabsf(cosine);
        hflags |= 8u | 2u;
    }
    if (vdot(dir, fn) < 0.0f && count_emitted) L = vadd(L, vmul(thr, emis));
    if (emis.x + emis.y + emis.z > 0.0f) hflags |= 16u;
    out->position = position;
    out->direction = direction;
    out->cur_thr = cur_thr;
    out->bsdf_val = bsdf_val;
    out->L = L;
    out->cosine = cosine;
    out->wo_pdf = wo_pdf;
    out->hflags = hflags;
    out->cell = cell;
    *prng = rng;
}

/* One sample per pixel for pixels [p0, p1) of the frame; accum += color (double), seeds
 * updated.  tree: an or_sdtree handle or NULL.  Returns the number of paths traced. */
static uint32_t* g_depth_out = NULL;
static int64_t g_log_pixel = -1;
static float* g_log = NULL; /* per bounce: org xyz, dir xyz, t, prim (as float bits) */
/* log the rays of one pixel (debugging aid) */
void or_render_log_pixel(int64_t pixel, float* out) { g_log_pixel = pixel; g_log = out; }
/* where or_render writes the final bounce index of every path (NULL = nowhere) */
void or_render_depth_output(uint32_t* out) { g_depth_out = out; }

int64_t or_render(const OScene* s, uint32_t flags, void* tree_h, void* grid_h, uint32_t p0, uint32_t p1,
                  uint32_t* seeds, double* accum) {
    OSDTree* tree = (OSDTree*)tree_h;
    OGrid* grid = (OGrid*)grid_h;
    const int use_tree = (flags & O_TREE) != 0, use_grid = (flags & O_GRID) != 0;
    const int recording = (use_tree || use_grid) && !(flags & O_FINAL);
    for (uint32_t p = p0; p < p1; ++p) {
        uint32_t x = p % s->width, y = p / s->width;
        uint32_t rng = seeds[p];
        float jx = rnd1(&rng), jy = rnd1(&rng);
        float dx = (2.0f * ((float)x + jx) / (float)s->width) - 1.0f;
        float dy = (2.0f * ((float)y + jy) / (float)s->height) - 1.0f;
        V3 cu = v3(s->cu[0], s->cu[1], s->cu[2]), cv = v3(s->cv[0], s->cv[1], s->cv[2]), cw = v3(s->cw[0], s->cw[1], s->cw[2]);
        V3 org = v3(s->eye[0], s->eye[1], s->eye[2]);
        V3 dir = vunit(vadd(vadd(vs(dx, cu), vs(dy, cv)), cw));
        V3 thr = v3(1, 1, 1), col = v3(0, 0, 0);
        uint32_t pflags = 8u /* COUNT_EMITTED */, depth = 0;
        OVert verts[O_KTV];
        for (;;) {
            uint32_t tvd = depth < O_KTV ? depth : O_KTV;
            float t = 0, hu = 0, hv = 0;
            uint32_t prim = 0;
            V3 L = v3(0, 0, 0), cur_thr = thr, direction = v3(0, 0, 0), bsdf_val = v3(0, 0, 0);
            float cosine = 0.0f, wo_pdf = 0.0f;
            uint32_t hflags = 0;
            V3 position = org;
            int hit = o_trace(s, org, dir, 0.0001f, 1.0e20f, 0, &t, &prim, &hu, &hv);
            if ((int64_t)p == g_log_pixel && g_log && depth < 16) {
                float* lg = g_log + 8 * depth;
                lg[0] = org.x; lg[1] = org.y; lg[2] = org.z; lg[3] = dir.x; lg[4] = dir.y; lg[5] = dir.z;
                lg[6] = hit ? t : -1.0f;
                uint32_t pb = hit ? prim : 0xffffffffu;
                memcpy(&lg[7], &pb, 4);
            }
            if (!hit) {
                L = vmul(thr, v3(s->bg[0], s->bg[1], s->bg[2]));
                hflags = 16u;
                if (recording && depth < O_KTV) verts[depth].valid = 0;
            } else {
                OShade sh;
                o_shade(s, flags, tree, grid, org, dir, t, prim, hu, hv, thr, pflags, depth, &rng, &sh);
                position = sh.position;
                direction = sh.direction;
                cur_thr = sh.cur_thr;
                bsdf_val = sh.bsdf_val;
                L = sh.L;
                cosine = sh.cosine;
                wo_pdf = sh.wo_pdf;
                hflags = sh.hflags;
                const uint32_t cell = sh.cell;
                if (recording && depth < O_KTV) {
                    OVert* v = &verts[depth];
                    v->pos = position; v->dir = direction; v->thr = cur_thr; v->rad = v3(0, 0, 0);
                    v->bsdf = bsdf_val; v->wopdf = wo_pdf; v->cosine = cosine; v->delta = (hflags & 2u) != 0;
                    v->valid = use_grid ? cell != UINT32_MAX : 1;
                    v->cell = cell;
                }
            }
            if (recording)
                for (uint32_t i = 0; i < tvd; ++i) verts[i].rad = vadd(verts[i].rad, L);
            col = vadd(col, L);
            org = position;
            dir = direction;
            thr = cur_thr;
            pflags = hflags;
            if (vnan(dir) || vnan(thr) || vnan(L)) break;
            if ((hflags & 16u) || depth >= s->max_depth - 1) break;
            ++depth;
        }
        if (recording) {
            uint32_t nv = depth < O_KTV ? depth : O_KTV;
            for (uint32_t i = 0; i < nv; ++i) {
                if (use_grid) commit_vertex_grid(grid, &verts[i]);
                else commit_vertex(tree, &verts[i]);
            }
        }
        if (g_depth_out) g_depth_out[p] = depth;
        accum[3 * (size_t)p] += col.x;
        accum[3 * (size_t)p + 1] += col.y;
        accum[3 * (size_t)p + 2] += col.z;
        seeds[p] = rng;
    }
    return (int64_t)(p1 - p0);
}

/* ------------------------------------------------------------------ known answers
 * The integrator's building blocks one call at a time, for the known-answer tests that pin
 * them against RTLib's own code run on the host (oracle/ref) and against the golden
 * fixture it wrote.  Xorshift32 states are in/out (one per case). */
void or_kat_cosine(int64_t n, const float* normal, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 d = o_sample_cosine(v3(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]), &state[i]);
        out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
    }
}
void or_kat_phong(int64_t n, const float* refl, const float* shininess, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 d = o_sample_phong(v3(refl[3 * i], refl[3 * i + 1], refl[3 * i + 2]), shininess[i], &state[i]);
        out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
    }
}
void or_kat_triangle(int64_t n, const float* v, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* q = v + 9 * i;
        V3 p = o_random_in_unit_triangle(v3(q[0], q[1], q[2]), v3(q[3], q[4], q[5]), v3(q[6], q[7], q[8]), &state[i]);
        out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
    }
}
/* nseq sequences of len updates: weights w[nseq][len], uniforms rnd[nseq][len]; per sequence
 * the index last kept (-1: none), w_sum and m */
void or_kat_reservoir(int64_t nseq, int32_t len, const float* w, const float* rnd, int32_t* sel, float* wsum,
                      uint32_t* m) {
    for (int64_t k = 0; k < nseq; ++k) {
        float ws = 0.0f;
        uint32_t mm = 0;
        int32_t y = -1;
        for (int32_t i = 0; i < len; ++i)
            if (o_reservoir_update(&ws, &mm, w[k * len + i], rnd[k * len + i])) y = i;
        sel[k] = y;
        wsum[k] = ws;
        m[k] = mm;
    }
}
/* per case 14 floats: direction, normal, emission, distance, invPdf, position */
void or_kat_light(const OScene* s, int64_t n, const float* p_in, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 pin = v3(p_in[3 * i], p_in[3 * i + 1], p_in[3 * i + 2]);
        OLight l = o_sample_light(s, pin, &state[i]);
        float* o = out + 14 * i;
        V3 pos = l.pos;
        o[0] = l.dir.x; o[1] = l.dir.y; o[2] = l.dir.z;
        o[3] = l.normal.x; o[4] = l.normal.y; o[5] = l.normal.z;
        o[6] = l.emission.x; o[7] = l.emission.y; o[8] = l.emission.z;
        o[9] = l.dist; o[10] = l.inv_pdf;
        o[11] = pos.x; o[12] = pos.y; o[13] = pos.z;
    }
}
/* o_shade of n vertices: the ray (org, dir), hit distance t and triangle prim, throughput,
 * previous hit flags and depth of each; per case 17 floats out (position, direction,
 * throughput after the vertex, BSDF value, radiance added, cosine, woPdf) and the hit flags.
 * tree: an or_sdtree handle (USE_TREE) or NULL. */
void or_kat_shade(const OScene* s, uint32_t flags, void* tree, int64_t n, const float* org, const float* dir,
                  const float* t, const uint32_t* prim, const float* thr, const uint32_t* pflags, const uint32_t* depth,
                  uint32_t* state, float* out, uint32_t* out_flags) {
    for (int64_t i = 0; i < n; ++i) {
        OShade sh;
        o_shade(s, flags, (OSDTree*)tree, NULL, v3(org[3 * i], org[3 * i + 1], org[3 * i + 2]),
                v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]), t[i], prim[i], 0.0f, 0.0f,
                v3(thr[3 * i], thr[3 * i + 1], thr[3 * i + 2]), pflags[i], depth[i], &state[i], &sh);
        float* o = out + 17 * i;
        const V3* vv[5] = {&sh.position, &sh.direction, &sh.cur_thr, &sh.bsdf_val, &sh.L};
        for (int k = 0; k < 5; ++k) { o[3 * k] = vv[k]->x; o[3 * k + 1] = vv[k]->y; o[3 * k + 2] = vv[k]->z; }
        o[15] = sh.cosine;
        o[16] = sh.wo_pdf;
        out_flags[i] = sh.hflags;
    }
}
