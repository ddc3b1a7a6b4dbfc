// Wavefront path tracer with SD-tree guiding, NEE and RIS (rtpg_tracer_*).
//
// RTLib renders with OptiX megakernels: __raygen__default loops over bounces and keeps up to
// 10 trace vertices per path (SimpleGuide.cu:48-156); __closesthit__radiance shades, samples
// the BSDF / guide mixture and does NEE or RIS with one shadow ray (SimpleGuide.cu:287-520,
// SimpleTrace.cu for the unguided tracers).  Here the same per-path algorithm runs as a
// wavefront over SoA path state, one frame of paths (one sample per pixel) per wave:
//   raygen   camera rays, per-pixel Xorshift32 state from the seed buffer;
//   bounce   closest hit + shading of every active path: emission, BSDF / guide mixture
//            sampling, NEE or RIS candidate selection and its shadow ray, the bounce radiance
//            added to the path, termination, compaction of survivors into the next queue;
//   finish   accumulation in FP64, seed write-back, and the commit of trace vertices into
//            the SD-tree (TraceVertexT::Commit, OPX7UtilsPathGuiding.h:830-866) with the
//            fixed-point atomics of the record kernel.
// A wave is captured once per configuration into a CUDA graph and replayed per sample.
#include <map>
#include <string.h>
#include <new>
#include <vector>

#include "common.cuh"
#include "bvh_dev.cuh"
#include "hashgrid_dev.cuh"
#include "mlp_dev.cuh"
#include "mqt_dev.cuh"
#include "sdtree_dev.cuh"
#include "tracer_dev.cuh"

struct rtpg_scene;
struct rtpg_sdtree;
struct rtpg_hashgrid;
struct rtpg_mqt;
struct rtpg_mlp;
namespace rtpg {
MlpView mlp_view(const rtpg_mlp* h);
SceneDev scene_device_view(const rtpg_scene* s);
SDTreeDev sdtree_device_view(const rtpg_sdtree* t);
HashGridDev hashgrid_device_view(const rtpg_hashgrid* h);
MqtDev mqt_device_view(const rtpg_mqt* h);
}

namespace rtpg {

constexpr int kTV = 10;  // trace vertices per path (kTraceVertexSize, OPX7/CMakeLists.txt:90)
constexpr int kTB = 128;

struct TracerDev {
    SceneDev scene;
    const float* tri_v;     // 9 floats per triangle (original order)
    const TriFrame* tri_frame;  // per triangle: face normal, half area, the normal's ONB
    const float* tri_uv;    // 6 floats per triangle or null
    const uint32_t* tri_mat;
    const Material* mats;
    const float* const* tex;  // per texture: RGB float, tex_wh[t] = (w, h)
    const uint2* tex_wh;
    const uint32_t* light_tris;
    const uint2* light_mesh;  // (first, count) into light_tris
    const float3* light_emit;
    uint32_t light_count;
    uint32_t num_materials, num_light_tris;
    float3 eye, cu, cv, cw, bg;
    uint32_t width, height, npath, max_depth, num_candidates, flags;
    // path state
    float3 *org, *dir, *thr, *col;
    uint32_t *rng, *depth, *hflags;
    uint32_t* queue[2];
    // queue lengths, three in rotation: bounce b reads [b % 3], appends to [(b + 1) % 3] and
    // zeroes [(b + 2) % 3], which no block of that launch touches
    uint32_t* qcount;
    // trace vertices, [kTV][npath]
    float3 *v_pos, *v_dir, *v_thr;
    float3* b_rad;  // radiance of bounce k of every path, [max_depth][npath] (recording only)
    float *v_wopdf, *v_cos;
    uint8_t* v_flags;  // bit0 valid (a DTree exists / a grid cell was found), bit1 delta
    uint32_t* v_cell;  // hash-grid slot (grid guide) or DTree (SD-tree guide) of the vertex
    // where the commit adds the vertex's radiance: the building-quadtree quadrant (SD-tree) or
    // the Morton leaf code inside the cell's tree (grid), found while the direction is at hand
    uint32_t* v_slot;
    uint32_t* seeds;
    double* accum;  // 3 per pixel
    SDTreeDev tree;
    HashGridDev grid;
    MqtDev mqt;
    unsigned* status;
    unsigned long long* counters;  // [0] bounce visits (path-bounces), [1] shadow rays
    // adjoint replay (path-replay backpropagation)
    const float3* adj_c;   // radiance of every path from the primal replay of this sample
    float3* lrem;          // radiance still ahead of the path during the adjoint replay
    const float* adj_dimg; // dLoss/dImage, RGB per pixel
    float adj_scale;       // 1 / samples of the image
    int32_t adj_tex;       // texture whose texels get gradients (-1: none)
    float* grad_tex;       // 3 per texel of adj_tex
    float* grad_light;     // 3 per light mesh
    const int32_t* mat_light;  // light mesh of an emissive material, -1 otherwise
    // learned guide: hits found ahead of shading, the mixture of every path, record appends
    MlpView ml;
    float mlp_fraction, mlp_keep, mlp_share;
    uint32_t* hit_prim;
    float4* hit_tuv;
    __half* lobes;  // 40 per path: 8 x (mu xyz, kappa, weight)
    float3 *v_nrm, *v_wo;
    // A scene of at most kFlatTris triangles travels inside the kernel parameters: every lane
    // tests the same triangle at the same time, so its rows are read from the constant bank
    // with no load instruction, no load latency and no vector registers holding them.
    uint32_t nflat;  // 0: trace through the BVH
    BvhTri ftri[kFlatTris];
};

// closest hit (ANY = false) or any hit (ANY = true) in (tmin, tmax): the scene's triangles from
// the kernel parameters when it is small, else the BVH
template <bool ANY>
__device__ __forceinline__ Hit trace(const TracerDev& T, float ox, float oy, float oz, float dx, float dy, float dz,
                                     float tmin, float tmax) {
    if (T.nflat) return flat_trace<ANY>(T.ftri, T.nflat, ox, oy, oz, dx, dy, dz, tmin, tmax);
    return bvh_trace<ANY>(T.scene, ox, oy, oz, dx, dy, dz, tmin, tmax);
}

// ------------------------------------------------------------------ raygen (SimpleGuide.cu:48-81)
__global__ void __launch_bounds__(kTB) k_raygen(TracerDev T) {
    grid_dependency_wait();  // the wave's kernels are dependent launches (see launch_wave)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        T.qcount[0] = T.npath;  // bounce 0 reads [0], appends to [1], zeroes [2]
        T.qcount[1] = 0;
    }
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < T.npath; p += gridDim.x * blockDim.x) {
        const uint32_t x = p % T.width, y = p / T.width;
        uint32_t rng = T.seeds[p];
        const float jx = rnd1(rng);
        const float jy = rnd1(rng);
        const float dx = (2.0f * ((float)x + jx) / (float)T.width) - 1.0f;
        const float dy = (2.0f * ((float)y + jy) / (float)T.height) - 1.0f;
        T.org[p] = T.eye;
        T.dir[p] = unit3(dx * T.cu + dy * T.cv + T.cw);
        T.thr[p] = f3(1.0f, 1.0f, 1.0f);
        T.col[p] = f3(0.0f, 0.0f, 0.0f);
        T.rng[p] = rng;
        T.depth[p] = 0;
        T.hflags[p] = HF_COUNT_EMITTED;
        T.queue[0][p] = p;
        if (T.adj_c) T.lrem[p] = T.adj_c[p];
    }
}

__device__ __forceinline__ float3 tex_fetch(const TracerDev& T, int t, float u, float v, uint32_t& texel) {
    const uint2 wh = T.tex_wh[t];
    float fu = u - floorf(u), fv = v - floorf(v);
    uint32_t x = min((uint32_t)(fu * wh.x), wh.x - 1), y = min((uint32_t)(fv * wh.y), wh.y - 1);
    texel = y * wh.x + x;
    const float* px = T.tex[t] + 3 * size_t(texel);
    return f3(px[0], px[1], px[2]);
}

struct LightSample {
    float3 pos, dir, normal, emission;
    float dist, inv_pdf;
    uint32_t mesh;
};
// MeshLightList::Sample -> MeshLight::Sample (SimpleKernel.h:81-98, 114-120): mesh and
// triangle by next() % count, barycentrics by random_in_unit_triangle.
__device__ __forceinline__ LightSample sample_light(const TracerDev& T, float3 p_in, uint32_t& rng) {
    const uint32_t mi = xs32_next(rng) % T.light_count;
    const uint2 mesh = T.light_mesh[mi];
    const uint32_t ti = min(T.light_tris[mesh.x + xs32_next(rng) % mesh.y], T.scene.ntris - 1);
    const float* tv = T.tri_v + 9 * size_t(ti);
    const float3 v0 = f3(tv[0], tv[1], tv[2]), v1 = f3(tv[3], tv[4], tv[5]), v2 = f3(tv[6], tv[7], tv[8]);
    const float4 f0 = T.tri_frame[ti].fr[0];  // unit3(cross(v1 - v0, v2 - v0)), half its length
    const float r0 = rnd1(rng);
    const float r1 = rnd1(rng);
    const float a = fminf(r0, r1), b = fmaxf(r0, r1);
    const float3 p = a * v0 + (1.0f - b) * v1 + (b - a) * v2;
    const float3 d = p - p_in;
    LightSample l;
    l.pos = p;
    l.dist = len3(d);
    l.dir = unit3(d);
    l.emission = T.light_emit[mi];
    l.normal = xyz(f0);
    l.inv_pdf = f0.w * (float)mesh.y * (float)T.light_count;
    l.mesh = mi;
    return l;
}

// ------------------------------------------------------------------ bounce
// One bounce of every active path: closest hit + shading (__closesthit__radiance /
// __miss__radiance, SimpleGuide.cu:202-520), the NEE/RIS shadow ray traced right away as the
// closest-hit program does, then the raygen bookkeeping (SimpleGuide.cu:85-114): bounce
// radiance into the color (and, recording, into the per-bounce store from which k_commit forms
// the trace-vertex radiance), termination, compaction of the survivors into the next queue.
// Returns whether the path continues; *shadow tells whether a shadow ray was traced.
constexpr int kGuideNone = 0, kGuideTree = 1, kGuideGrid = 2, kAdjoint = 3, kGuideMlp = 4;

// The adjoint replay (kAdjoint) runs the unguided path again from the same random numbers and
// scatters d(loss)/d(parameter) as it goes (path-replay backpropagation): lrem starts as the
// path's radiance from the primal replay and loses each term once the path has passed it, so
// at a textured vertex it holds exactly the terms that carry the vertex's albedo as a factor
// (its NEE term and everything after it); the albedo gradient is delta * lrem / albedo per
// channel.  An emitter's gradient is delta * (the term's factor in front of its radiance).
template <int G>
__device__ __forceinline__ bool bounce_path(const TracerDev& T, uint32_t p, bool build, bool recording, bool& shadow) {
    constexpr bool use_tree = G == kGuideTree, use_grid = G == kGuideGrid, adjoint = G == kAdjoint;
    constexpr bool use_mlp = G == kGuideMlp;
    const float3 org = T.org[p], in_dir = T.dir[p], prev_thr = T.thr[p];
    const uint32_t d = T.depth[p], prev_flags = T.hflags[p];
    Hit h;
    if (use_mlp) {  // found by k_hit ahead of the mixture inference
        const float4 tuv = T.hit_tuv[p];
        h.prim = T.hit_prim[p];
        h.t = tuv.x;
        h.u = tuv.y;
        h.v = tuv.z;
    } else {
        h = trace<false>(T, org.x, org.y, org.z, in_dir.x, in_dir.y, in_dir.z, 0.0001f, 1.0e20f);
    }
    const size_t vi = size_t(d < kTV ? d : 0) * T.npath + p;
    bool pend = false;
    float3 sdir = f3(0.f, 0.f, 0.f), scontrib = f3(0.f, 0.f, 0.f);
    float sdist = 0.0f;
    uint32_t nee_mesh = 0xffffffffu;                 // adjoint: light mesh of the NEE sample
    float3 nee_factor = f3(0.f, 0.f, 0.f);           // adjoint: NEE term / light radiance
    if (h.prim == 0xffffffffu) {
        // __miss__radiance (SimpleGuide.cu:202-219): the ray keeps its direction
        const float3 L = prev_thr * T.bg;
        if (recording) T.b_rad[size_t(d) * T.npath + p] = L;
        T.col[p] = T.col[p] + L;
        if (recording && d < kTV) T.v_flags[vi] = 0;
        return false;
    }
    uint32_t rng = T.rng[p];
    const TriFrame& tf = T.tri_frame[h.prim];
    const float3 fn = xyz(tf.fr[0]);
    float3 position = org + h.t * in_dir;
    const uint32_t mi = T.tri_mat[h.prim];
    const Material m = T.mats[mi < T.num_materials ? mi : T.num_materials - 1];
    float3 diffuse = m.diffuse, texv = f3(1.f, 1.f, 1.f);
    uint32_t texel = 0xffffffffu;
    if (m.tex >= 0 && T.tri_uv) {
        const float* uv = T.tri_uv + 6 * size_t(h.prim);
        const float w0 = 1.0f - h.u - h.v;
        const float tu = w0 * uv[0] + h.u * uv[2] + h.v * uv[4];
        const float tvv = w0 * uv[1] + h.u * uv[3] + h.v * uv[5];
        texv = tex_fetch(T, m.tex, tu, tvv, texel);
        diffuse = diffuse * texv;
        if (adjoint && m.tex != T.adj_tex) texel = 0xffffffffu;
    }
    const bool count_emitted = (prev_flags & HF_COUNT_EMITTED) || m.type == MAT_DEF_LIGHT;
    float3 direction = f3(0.f, 0.f, 0.f), bsdf_val = f3(0.f, 0.f, 0.f), cur_thr = f3(0.f, 0.f, 0.f);
    float cosine = 0.0f, bsdf_pdf = 0.0f, wo_pdf = 0.0f;
    uint32_t flags = 0;
    uint32_t dt = 0;
    uint32_t cell = 0xffffffffu;  // hash-grid slot of this vertex (SimpleGuide2.cu: curGridIndex)
    float2 cdir = make_float2(0.f, 0.f);  // dir_to_canonical(direction), once the guide formed it
    bool have_c = false;
    // the learned guide may carry the SD-tree as its fallback (T.tree set, mlp_share < 1)
    const bool mlp_mix = use_mlp && T.tree.snode != nullptr;
    if (use_tree || mlp_mix) dt = stree_lookup(T.tree.snode, T.tree.mn, T.tree.mx, position.x, position.y, position.z, T.tree.inv_size,
                                                 T.tree.stop);
    if (m.type == MAT_PHONG) {
        uint32_t gbucket = 0, prv_cell = 0xffffffffu;
        unsigned long long gkey = 0;
        if (use_grid) {
            gkey = hash_key(T.grid, position.x, position.y, position.z, gbucket);
            prv_cell = hash_find_prv_key(T.grid, gkey, gbucket);
        }
        // With specular == 0 (every Lambertian surface) the Phong lobe only ever enters
        // multiplied by zero: skip its math but draw its two random numbers, so the stream
        // and every result stay bit-identical to the full evaluation.
        const float ad = 1.0e-10f + avg3(diffuse), as = 1.0e-10f + avg3(m.specular);
        const float sel = ad / (ad + as);
        // (sel == 1 as well: then the lobe choice and the pdf mixture never use it either)
        const bool glossy = m.specular.x != 0.0f || m.specular.y != 0.0f || m.specular.z != 0.0f || sel != 1.0f;
        // the mirror direction only enters glossy shading (its normalisation is a square root
        // and three divisions)
        const float3 refl = glossy ? unit3(reflect3(in_dir, fn)) : f3(0.f, 0.f, 1.f);
        const float3 d0 = sample_cosine(Onb(xyz(tf.fr[2]), xyz(tf.fr[3]), xyz(tf.fr[1])), rng);
        float3 d1 = d0;
        if (glossy) {
            d1 = sample_phong(refl, m.shininess, rng);
        } else {
            xs32_next(rng);
            xs32_next(rng);
        }
        const float c0 = dot3(d0, fn), c1 = dot3(d1, fn);
        const float cp0 = fmaxf(c0 * kInvPi, 0.0f), cp1 = fmaxf(c1 * kInvPi, 0.0f);
        const float pp0 = glossy ? phong_pdf(d0, refl, m.shininess) : 0.0f;
        const float pp1 = glossy ? phong_pdf(d1, refl, m.shininess) : 0.0f;
        const float sf = (m.shininess + 2.0f) / (m.shininess + 1.0f);
        if (rnd1(rng) < sel) {
            direction = d0; cosine = c0;
            bsdf_val = diffuse * kInvPi + m.specular * sf * pp0;
            bsdf_pdf = sel * cp0 + (1.0f - sel) * pp0;
        } else {
            direction = d1; cosine = c1;
            bsdf_val = diffuse * kInvPi + m.specular * sf * pp1;
            bsdf_pdf = sel * cp1 + (1.0f - sel) * pp1;
        }
        if (use_tree && build) {
            const uint32_t soff = T.tree.s_off[dt];
            const bool guided = T.tree.s_guided[dt] != 0;
            // square + pdf of a guided sample; the empty default sends the pdf of a BSDF sample
            // through the full descent
            DSquare sq{2.0f, 2.0f, 0.0f, 0.0f};
            if (rnd1(rng) < T.tree.fraction) {
                const float2 c = dtree_sample_sq(T.tree.s_q, T.tree.s_fac, soff, guided, rng, sq);
                direction = normalize3(canonical_to_dir(c.x, c.y));
                cosine = dot3(direction, fn);
                const float cp2 = fmaxf(cosine * kInvPi, 0.0f);
                const float pp2 = glossy ? phong_pdf(direction, refl, m.shininess) : 0.0f;
                bsdf_val = diffuse * kInvPi + m.specular * sf * pp2;
                bsdf_pdf = sel * cp2 + (1.0f - sel) * pp2;
            }
            const float2 c = dir_to_canonical(direction.x, direction.y, direction.z);
            cdir = c;
            have_c = true;
            const float dtree_pdf = fmaxf(dtree_pdf_in(T.tree.s_q, T.tree.s_fac, soff, guided, sq, c.x, c.y), 0.0f);
            wo_pdf = (1.0f - T.tree.fraction) * bsdf_pdf + T.tree.fraction * dtree_pdf;
        } else if (use_mlp && build) {
            // the learned mixture of this path's hit (k_mlp_lobes)
            VmfLobe Lb[kMlpLobes];
            {
                // 80 bytes per path: five 16-byte loads
                __align__(16) __half lp[40];
                const uint4* src = reinterpret_cast<const uint4*>(T.lobes + size_t(p) * 40);
#pragma unroll
                for (int k = 0; k < 5; ++k) reinterpret_cast<uint4*>(lp)[k] = src[k];
#pragma unroll
                for (int k = 0; k < kMlpLobes; ++k) {
                    Lb[k].mu = f3(__half2float(lp[5 * k]), __half2float(lp[5 * k + 1]), __half2float(lp[5 * k + 2]));
                    Lb[k].kappa = __half2float(lp[5 * k + 3]);
                    Lb[k].weight = __half2float(lp[5 * k + 4]);
                }
            }
            // guide density q = share * network + (1 - share) * SD-tree (the fallback)
            uint32_t soff = 0;
            bool tguided = false;
            if (mlp_mix) {
                soff = T.tree.s_off[dt];
                tguided = T.tree.s_guided[dt] != 0;
            }
            DSquare sq{2.0f, 2.0f, 0.0f, 0.0f};  // as in the SD-tree guide above
            if (rnd1(rng) < T.mlp_fraction) {
                if (!mlp_mix || rnd1(rng) < T.mlp_share) {
                    const float u0 = rnd1(rng);
                    const float u1 = rnd1(rng);
                    const float u2 = rnd1(rng);
                    direction = normalize3(vmf_mixture_sample(Lb, u0, u1, u2));
                } else {
                    const float2 c = dtree_sample_sq(T.tree.s_q, T.tree.s_fac, soff, tguided, rng, sq);
                    direction = normalize3(canonical_to_dir(c.x, c.y));
                }
                cosine = dot3(direction, fn);
                const float cp2 = fmaxf(cosine * kInvPi, 0.0f);
                const float pp2 = glossy ? phong_pdf(direction, refl, m.shininess) : 0.0f;
                bsdf_val = diffuse * kInvPi + m.specular * sf * pp2;
                bsdf_pdf = sel * cp2 + (1.0f - sel) * pp2;
            }
            float q = vmf_mixture_pdf(Lb, direction);
            if (mlp_mix) {
                const float2 c = dir_to_canonical(direction.x, direction.y, direction.z);
                cdir = c;
                have_c = true;
                const float qt = fmaxf(dtree_pdf_in(T.tree.s_q, T.tree.s_fac, soff, tguided, sq, c.x, c.y), 0.0f);
                q = T.mlp_share * q + (1.0f - T.mlp_share) * qt;
            }
            wo_pdf = (1.0f - T.mlp_fraction) * bsdf_pdf + T.mlp_fraction * q;
        } else if (use_grid && build && prv_cell != 0xffffffffu) {
            // the Morton quadtree of the cell (SimpleGuide2.cu:350-377)
            float dtree_pdf;
            if (rnd1(rng) < T.mqt.fraction) {
                float tp;
                const float2 c = mqt_sample_and_pdf(T.mqt, prv_cell, rng, tp);
                dtree_pdf = (float)((double)tp * (0.25 * kInvPiD));
                direction = normalize3(canonical_to_dir(c.x, c.y));
                cosine = dot3(direction, fn);
                const float cp2 = fmaxf(cosine * kInvPi, 0.0f);
                const float pp2 = glossy ? phong_pdf(direction, refl, m.shininess) : 0.0f;
                bsdf_val = diffuse * kInvPi + m.specular * sf * pp2;
                bsdf_pdf = sel * cp2 + (1.0f - sel) * pp2;
            } else {
                const float2 c = dir_to_canonical(direction.x, direction.y, direction.z);
                cdir = c;
                have_c = true;
                const float tp = mqt_pdf(T.mqt, prv_cell, c.x, c.y);
                dtree_pdf = fmaxf((float)((double)(tp * 0.25f) * kInvPiD), 0.0f);
            }
            wo_pdf = T.mqt.fraction * dtree_pdf + (1.0f - T.mqt.fraction) * bsdf_pdf;
        } else {
            wo_pdf = bsdf_pdf;
        }
        cur_thr = prev_thr * ((wo_pdf > 0.0f) ? (bsdf_val * fmaxf(cosine, 0.0f) / wo_pdf) : f3(0.f, 0.f, 0.f));
        if (T.flags & RTPG_TRACE_FLAG_NEE) {
            if (d < T.max_depth - 1 && T.light_count > 0) {
                if (T.flags & RTPG_TRACE_FLAG_RIS) {
                    // RIS over numCandidates light samples (SimpleGuide.cu:379-408)
                    float w_sum = 0.0f, f_a_y = 0.0f, dist_y = 0.0f;
                    uint32_t mcount = 0;
                    float3 f_y = f3(0.f, 0.f, 0.f), ldir_y = f3(0.f, 0.f, 0.f);
                    for (uint32_t c = 0; c < T.num_candidates; ++c) {
                        const LightSample l = sample_light(T, position, rng);
                        const float ndl = dot3(l.dir, fn), lndl = -dot3(l.dir, l.normal);
                        const float3 b = glossy ? phong_bsdf(diffuse, m.specular, m.shininess, l.dir, refl)
                                                : diffuse * kInvPi;
                        const float g = fmaxf(ndl, 0.0f) * fmaxf(lndl, 0.0f) / (l.dist * l.dist);
                        const float3 f = b * l.emission * g;
                        const float fa = avg3(f);
                        const float wi = fa * l.inv_pdf;
                        // Reservoir::Update (SimpleKernel.h:124-143)
                        w_sum += wi;
                        ++mcount;
                        if ((wi / w_sum) >= rnd1(rng)) {
                            f_y = f; f_a_y = fa; ldir_y = l.dir; dist_y = l.dist;
                        }
                    }
                    if (w_sum > 0.0f && f_a_y > 0.0f) {
                        pend = true;
                        sdir = ldir_y;
                        sdist = dist_y - 0.0001f;
                        scontrib = prev_thr * f_y * (w_sum / (f_a_y * (float)mcount));
                    }
                } else {
                    // one light sample (SimpleGuide.cu:410-419)
                    const LightSample l = sample_light(T, position, rng);
                    const float3 b = glossy ? phong_bsdf(diffuse, m.specular, m.shininess, l.dir, refl)
                                            : diffuse * kInvPi;
                    const float g = fmaxf(-dot3(l.dir, l.normal), 0.0f) * fabsf(dot3(l.dir, fn)) / (l.dist * l.dist);
                    pend = true;
                    sdir = l.dir;
                    sdist = l.dist - 0.0001f;
                    scontrib = prev_thr * b * l.emission * g * l.inv_pdf;
                    if (adjoint) {
                        nee_mesh = l.mesh;
                        nee_factor = prev_thr * b * g * l.inv_pdf;
                    }
                }
            }
        } else {
            flags |= HF_COUNT_EMITTED;
        }
        if (use_grid)
            cell = ((T.flags & RTPG_TRACE_FLAG_LOCATE) && prv_cell == 0xffffffffu) ? hash_insert_cur_key(T.grid, gkey, gbucket)
                                                                                  : prv_cell;
    } else if (m.type == MAT_GLASS) {
        // dielectric (SimpleGuide.cu:424-491), shading normal = face normal
        float3 rn;
        float rri;
        float ci = dot3(fn, in_dir);
        if (ci < 0.0f) { rn = fn; rri = 1.0f / m.ref_index; ci = -ci; }
        else { rn = f3(-fn.x, -fn.y, -fn.z); rri = m.ref_index; }
        const float so2 = (1.0f - ci * ci) * (rri * rri);
        const float f0 = ((1.0f - rri) / (1.0f + rri)) * ((1.0f - rri) / (1.0f + rri));
        const float om = 1.0f - ci;
        const float fres = f0 + (1.0f - f0) * (om * om * om * om * om);
        const float3 rd = unit3(reflect3(in_dir, rn));
        if (rnd1(rng) < fres || so2 > 1.0f) {
            position = position + 0.0001f * rn;
            direction = rd;
            cosine = fabsf(ci);
            bsdf_val = m.specular;
            cur_thr = prev_thr * m.specular;
        } else {
            position = position - 0.0001f * rn;
            const float si2 = fmaxf(1.0f - ci * ci, 0.0f);
            const float co = sqrtf(1.0f - so2);
            float3 rf;
            if (si2 > 0.0f) {
                const float3 k = (in_dir + ci * rn) / sqrtf(si2);
                rf = unit3(sqrtf(so2) * k - co * rn);
            } else {
                rf = in_dir;
            }
            direction = rf;
            cosine = fabsf(dot3(rf, rn));
            bsdf_val = f3(1.f, 1.f, 1.f);
            cur_thr = prev_thr;
        }
        wo_pdf = fabsf(cosine);
        bsdf_pdf = 0.0f;
        flags |= HF_COUNT_EMITTED | HF_DELTA;
    }
    float3 rad = f3(0.f, 0.f, 0.f);
    const bool emitted = dot3(in_dir, fn) < 0.0f && count_emitted;
    if (emitted) rad = prev_thr * m.emission;
    if (m.emission.x + m.emission.y + m.emission.z > 0.0f) flags |= HF_FINISH;
    T.org[p] = position;
    T.dir[p] = direction;
    T.thr[p] = cur_thr;
    T.hflags[p] = flags;
    T.rng[p] = rng;
    if (recording && d < kTV) {
        if (use_mlp) {
            T.v_pos[vi] = position;
            T.v_dir[vi] = direction;
        }
        T.v_thr[vi] = cur_thr;
        T.v_wopdf[vi] = wo_pdf;
        T.v_cos[vi] = cosine;
        // bit 0: the commit may use the vertex -- a DTree / found cell, and a finite,
        // non-negative BSDF value (isValidBsdfVal of TraceVertexT::Commit); bit 1: delta
        const bool ok_b = isfinite(bsdf_val.x) && bsdf_val.x >= 0.f && isfinite(bsdf_val.y) && bsdf_val.y >= 0.f &&
                          isfinite(bsdf_val.z) && bsdf_val.z >= 0.f;
        const bool has_guide = use_grid ? cell != 0xffffffffu : true;
        T.v_flags[vi] = (uint8_t)((has_guide && ok_b ? 1u : 0u) | ((flags & HF_DELTA) ? 2u : 0u));
        if (use_grid) T.v_cell[vi] = cell;
        if (use_tree || mlp_mix) T.v_cell[vi] = dt;  // the vertex's DTree, found once here for the commit
        if ((use_tree || mlp_mix || use_grid) && !(flags & HF_DELTA)) {
            // canonical of the direction exactly as the commit would form it; the building
            // tree's topology does not change within a pass
            const float2 cr = have_c ? cdir : dir_to_canonical(direction.x, direction.y, direction.z);
            T.v_slot[vi] = use_grid ? mqt_leaf_code(T.mqt.level, cr.x, cr.y)
                                    : dtree_record_slot(T.tree.b_child, T.tree.b_off[dt], cr.x, cr.y);
        }
        if (use_mlp) {
            T.v_nrm[vi] = fn;
            T.v_wo[vi] = f3(-in_dir.x, -in_dir.y, -in_dir.z);
        }
    }
    float3 L = rad;
    bool lit = false;
    if (pend) {
        shadow = true;
        const Hit sh = trace<true>(T, position.x, position.y, position.z, sdir.x, sdir.y, sdir.z, 0.0001f, sdist);
        if (sh.prim == 0xffffffffu) {
            L = L + scontrib;
            lit = true;
        }
    }
    if (adjoint) {
        const float3 delta = f3(T.adj_dimg[3 * size_t(p)], T.adj_dimg[3 * size_t(p) + 1], T.adj_dimg[3 * size_t(p) + 2]) * T.adj_scale;
        float3 lr = T.lrem[p] - rad;  // the emission term does not depend on this vertex
        if (emitted) {
            const int32_t li = T.mat_light[mi < T.num_materials ? mi : T.num_materials - 1];
            if (li >= 0 && T.grad_light) {
                const float3 gl = delta * prev_thr;
                atomicAdd(T.grad_light + 3 * li, gl.x);
                atomicAdd(T.grad_light + 3 * li + 1, gl.y);
                atomicAdd(T.grad_light + 3 * li + 2, gl.z);
            }
        }
        if (texel != 0xffffffffu && T.grad_tex && m.type == MAT_PHONG) {
            // albedo enters the NEE term and the throughput linearly, per channel
            float* gt = T.grad_tex + 3 * size_t(texel);
            if (texv.x > 0.f) atomicAdd(gt, delta.x * lr.x / texv.x);
            if (texv.y > 0.f) atomicAdd(gt + 1, delta.y * lr.y / texv.y);
            if (texv.z > 0.f) atomicAdd(gt + 2, delta.z * lr.z / texv.z);
        }
        if (lit && nee_mesh != 0xffffffffu) {
            if (T.grad_light) {
                const float3 gl = delta * nee_factor;
                atomicAdd(T.grad_light + 3 * nee_mesh, gl.x);
                atomicAdd(T.grad_light + 3 * nee_mesh + 1, gl.y);
                atomicAdd(T.grad_light + 3 * nee_mesh + 2, gl.z);
            }
            lr = lr - scontrib;
        }
        T.lrem[p] = lr;
    }
    if (recording) T.b_rad[size_t(d) * T.npath + p] = L;
    T.col[p] = T.col[p] + L;
    const bool bad = any_nan3(direction) || any_nan3(cur_thr) || any_nan3(L);
    if (bad || (flags & HF_FINISH) || d >= T.max_depth - 1) return false;
    T.depth[p] = d + 1;
    if (use_mlp) {
        // the closest hit of the continuing ray, traced here rather than in a pass of its own,
        // so the network of the next bounce finds it waiting (k_hit serves the first bounce)
        const Hit nh = trace<false>(T, position.x, position.y, position.z, direction.x, direction.y,
                                        direction.z, 0.0001f, 1.0e20f);
        T.hit_prim[p] = nh.prim;
        T.hit_tuv[p] = make_float4(nh.t, nh.u, nh.v, 0.0f);
    }
    return true;
}

// guide kinds (and the adjoint replay), a template argument so that each variant carries only
// its own code
__host__ __device__ constexpr int guide_of(uint32_t flags) {
    return (flags & RTPG_TRACE_FLAG_USE_TREE) ? kGuideTree
           : (flags & RTPG_TRACE_FLAG_USE_GRID) ? kGuideGrid
           : (flags & RTPG_TRACE_FLAG_USE_MLP)  ? kGuideMlp
                                                 : kGuideNone;
}

// learned guide, stage 1 of the first bounce: closest hits of the camera rays (later bounces
// find theirs traced at the end of the previous k_bounce)
__global__ void __launch_bounds__(kTB) k_hit(TracerDev T, uint32_t bounce) {
    grid_dependency_wait();
    const int in = int(bounce & 1);
    const uint32_t n = T.qcount[bounce % 3];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t p = T.queue[in][q];
        const float3 o = T.org[p], d = T.dir[p];
        const Hit h = trace<false>(T, o.x, o.y, o.z, d.x, d.y, d.z, 0.0001f, 1.0e20f);
        T.hit_prim[p] = h.prim;
        T.hit_tuv[p] = make_float4(h.t, h.u, h.v, 0.0f);
    }
}

// learned guide, stage 2: the mixture of every queued path that hit a Phong surface, 128
// paths per tile on the tensor cores (features of path q in row q of the tile)
__global__ void __launch_bounds__(kMlpThreads) k_mlp_lobes(TracerDev T, uint32_t bounce) {
    grid_dependency_wait();
    const int in = int(bounce & 1);
    extern __shared__ __align__(128) uint8_t sm[];
    __nv_bfloat16* ws = reinterpret_cast<__nv_bfloat16*>(sm);
    __nv_bfloat16* x0 = reinterpret_cast<__nv_bfloat16*>(sm + kSmemW);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kSmemW + kSmemX);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmemW + kSmemX + 8);
    const int t = threadIdx.x;
    if (t < 32) tmem_alloc(tslot, kEvalCols);
    if (t == 0) mbar_init(mbar, 1);
    load_weights(ws, T.ml.dev.wq);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot, sw = smem_u32(ws);
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t n = T.qcount[bounce % 3];
    for (uint32_t base = blockIdx.x * kMlpTile; base < n; base += gridDim.x * kMlpTile) {
        const uint32_t q = base + t;
        bool live = false;
        uint32_t p = 0;
        float f[kMlpIn];
        if (q < n) {
            p = T.queue[in][q];
            const uint32_t prim = T.hit_prim[p];
            if (prim != 0xffffffffu) {
                const uint32_t mi = T.tri_mat[prim];
                live = T.mats[mi < T.num_materials ? mi : T.num_materials - 1].type == MAT_PHONG;
            }
            if (live) {
                const float4 tuv = T.hit_tuv[p];
                const float3 o = T.org[p], d = T.dir[p];
                const float3 fn = xyz(T.tri_frame[prim].fr[0]);
                mlp_features(o + tuv.x * d, fn, f3(-d.x, -d.y, -d.z), T.ml.dev.mn, T.ml.dev.inv_ext, f);
            }
        }
        if (!live)
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) f[k] = 0.0f;
        store_features(x0, t, f);
        float o[kMlpOut];
        if (!mlp_forward_tile(T.ml.dev, tmem, sw, x0, mbar, phase, o)) {
            ok = false;  // uniform over the CTA: issue nothing more
            break;
        }
        if (live) {
            VmfLobe L[kMlpLobes];
            mlp_head(o, L);
            __align__(16) __half lp[40];
#pragma unroll
            for (int k = 0; k < kMlpLobes; ++k) {
                lp[5 * k] = __float2half_rn(L[k].mu.x);
                lp[5 * k + 1] = __float2half_rn(L[k].mu.y);
                lp[5 * k + 2] = __float2half_rn(L[k].mu.z);
                lp[5 * k + 3] = __float2half_rn(L[k].kappa);
                lp[5 * k + 4] = __float2half_rn(L[k].weight);
            }
            // 80 bytes per path: five 16-byte stores
            uint4* dst = reinterpret_cast<uint4*>(T.lobes + size_t(p) * 40);
#pragma unroll
            for (int k = 0; k < 5; ++k) dst[k] = reinterpret_cast<const uint4*>(lp)[k];
        }
    }
    if (!ok) {
        if (t == 0) atomicOr(T.status, RTPG_STATUS_TIMEOUT);
        mma_drain(mbar, phase, T.ml.dev.poll_limit);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t < 32) tmem_dealloc(tmem, kEvalCols);
}

template <int G>
__global__ void __launch_bounds__(kTB, 8) k_bounce(TracerDev T, uint32_t bounce) {
    grid_dependency_wait();
    const int in = int(bounce & 1);
    uint32_t* const next_count = T.qcount + (bounce + 1) % 3;
    const uint32_t n = T.qcount[bounce % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        T.qcount[(bounce + 2) % 3] = 0;  // the next bounce's output
        atomicAdd(T.counters, (unsigned long long)n);
    }
    const bool build = (T.flags & RTPG_TRACE_FLAG_BUILD) != 0;
    const bool recording = (G == kGuideTree || G == kGuideGrid || G == kGuideMlp) && !(T.flags & RTPG_TRACE_FLAG_FINAL);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t q = base + threadIdx.x;
        bool keep = false, shadow = false;
        uint32_t p = 0;
        if (q < n) {
            p = T.queue[in][q];
            keep = bounce_path<G>(T, p, build, recording, shadow);
        }
        const unsigned sh = __ballot_sync(0xffffffffu, shadow);
        if ((threadIdx.x & 31) == 0 && sh) atomicAdd(T.counters + 1, (unsigned long long)__popc(sh));
        // warp-aggregated append to the next queue
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (m) {
            uint32_t base_q = 0;
            if (lane == __ffs(m) - 1) base_q = atomicAdd(next_count, (uint32_t)__popc(m));
            base_q = __shfl_sync(0xffffffffu, base_q, __ffs(m) - 1);
            if (keep) T.queue[in ^ 1][base_q + __popc(m & ((1u << lane) - 1u))] = p;
        }
    }
}

// ------------------------------------------------------------------ finish
// Per path: FP64 accumulation and the seed write-back.
__global__ void __launch_bounds__(kTB) k_finish(TracerDev T) {
    grid_dependency_wait();
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < T.npath; p += gridDim.x * blockDim.x) {
        const float3 c = T.col[p];
        double* a = T.accum + 3 * size_t(p);
        a[0] += (double)c.x;
        a[1] += (double)c.y;
        a[2] += (double)c.z;
        T.seeds[p] = T.rng[p];
    }
}

// The commit of the trace vertices of recording waves (TraceVertexT::Commit,
// OPX7UtilsPathGuiding.h:830-866 -> DTreeWrapperT::Record :514-520 with stat-weight 1, or
// MortonTraceVertexT::Commit for the grid guide), one thread per vertex: each CTA walks the
// vertex rows i = 0 .. kTV-1 over its share of the paths, so a warp holds vertex i of 32
// consecutive paths and lanes whose path is shorter leave at once.  The radiance of vertex i is
// L_{i+1} + L_{i+2} + ... added in bounce order, exactly the float sums RTLib's raygen loop
// accumulates into traceVertices[i].radiance (SimpleGuide.cu:98-100).
// Every committed vertex adds the same stat-weight to its DTree, a few hundred counters that
// millions of vertices hit: those adds go to a copy of the counters in the CTA's shared memory
// (up to kFinPrivTrees DTrees), flushed once per CTA; with kSMs * 2 CTAs of kCommitThreads the
// flush is a few hundred adds per counter instead of thousands of contended ones.  The
// quadrant sums go to shared memory too while the whole building tree is small (the first
// passes), else straight to the tree with 64-bit integer atomics: keys spread over thousands
// of nodes gain nothing from aggregation.
constexpr uint32_t kFinPrivQuads = 2048;
constexpr uint32_t kFinPrivTrees = 2048;
constexpr int kCommitThreads = 512;
template <int G>
__global__ void __launch_bounds__(kCommitThreads) k_commit(TracerDev T) {
    grid_dependency_wait();
    __shared__ unsigned long long s_q[kFinPrivQuads];
    __shared__ unsigned long long s_w[kFinPrivTrees];
    constexpr bool use_grid = G == kGuideGrid;
    // the learned guide with the SD-tree as fallback commits to both
    const bool tree_too = G == kGuideMlp && T.tree.snode != nullptr;
    const bool tree_commit = !use_grid && (G != kGuideMlp || tree_too);
    uint32_t nq = 0, ndt = 0;
    if (tree_commit) {
        nq = T.tree.counts[2] * 4u;
        ndt = T.tree.counts[1];
    }
    const bool priv_w = tree_commit && ndt <= kFinPrivTrees;
    const bool priv = priv_w && nq <= kFinPrivQuads;
    if (priv_w) {
        if (priv)
            for (uint32_t j = threadIdx.x; j < nq; j += blockDim.x) s_q[j] = 0ull;
        for (uint32_t j = threadIdx.x; j < ndt; j += blockDim.x) s_w[j] = 0ull;
        __syncthreads();
    }
    // vertex rows outside, paths inside: a warp-uniform loop (the grid guide's aggregated
    // atomics need the whole warp) over coalesced rows
    for (uint32_t i = 0; i < (uint32_t)kTV; ++i) {
    for (uint32_t base = blockIdx.x * blockDim.x; base < T.npath; base += gridDim.x * blockDim.x) {
        const uint32_t p = base + threadIdx.x;
        unsigned long long k_w = ~0ull, k_s = ~0ull, v_w = 0, v_s = 0;
        const uint32_t d = p < T.npath ? T.depth[p] : 0u;
        const size_t vi = size_t(i) * T.npath + p;
        const uint8_t vf = i < d ? T.v_flags[vi] : 0;
        if ((vf & 1) && !(vf & 2)) {
            // the vertex's data and the later bounces' radiances do not depend on one another:
            // all loads are issued before the first add (in-order issue would otherwise wait a
            // memory latency per bounce), then the radiances are added in bounce order
            const float wo_v = T.v_wopdf[vi];
            const float3 th = T.v_thr[vi];
            float3 rad = f3(0.f, 0.f, 0.f);
            for (uint32_t k0 = i + 1; k0 <= d; k0 += 8) {
                float3 Lk[8];
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j)
                    Lk[j] = (k0 + j <= d) ? T.b_rad[size_t(k0 + j) * T.npath + p] : f3(0.f, 0.f, 0.f);
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j)
                    if (k0 + j <= d) rad = rad + Lk[j];
            }
            const bool ok_r = isfinite(rad.x) && rad.x >= 0.f && isfinite(rad.y) && rad.y >= 0.f &&
                              isfinite(rad.z) && rad.z >= 0.f;
            const float wo = ok_r ? wo_v : 0.0f;
            if (wo > 0.0f) {
                float3 lr = f3(0.f, 0.f, 0.f);
                if (th.x * wo > 1e-4f) lr.x = rad.x / th.x;
                if (th.y * wo > 1e-4f) lr.y = rad.y / th.y;
                if (th.z * wo > 1e-4f) lr.z = rad.z / th.z;
                lr = lr * fabsf(T.v_cos[vi]);
                const float lavg = (lr.x + lr.y + lr.z) / 3.0f;
                const float irr = __fdiv_rn(lavg, wo);
                if (G == kGuideMlp) {
                    // a training record of the learned guide: the SD-tree's record with the
                    // vertex's normal and outgoing direction, kept with probability mlp_keep
                    if (isfinite(irr) && irr > 0.0f &&
                        to_uniform_float(pcg1d(T.rng[p] ^ (i * 0x9E3779B9u))) < T.mlp_keep) {
                        const uint32_t idx = atomicAdd(T.ml.r_count, 1u);
                        if (idx < T.ml.capacity) {
                            const float3 ps = T.v_pos[vi], nm = T.v_nrm[vi], wv = T.v_wo[vi], dr = T.v_dir[vi];
                            float* rp = T.ml.r_pos + 3 * size_t(idx);
                            float* rn = T.ml.r_nrm + 3 * size_t(idx);
                            float* ro = T.ml.r_wo + 3 * size_t(idx);
                            float* ri = T.ml.r_wi + 3 * size_t(idx);
                            rp[0] = ps.x; rp[1] = ps.y; rp[2] = ps.z;
                            rn[0] = nm.x; rn[1] = nm.y; rn[2] = nm.z;
                            ro[0] = wv.x; ro[1] = wv.y; ro[2] = wv.z;
                            ri[0] = dr.x; ri[1] = dr.y; ri[2] = dr.z;
                            T.ml.r_w[idx] = irr;
                            T.ml.r_pdf[idx] = wo;
                        }
                    }
                }
                if (G == kGuideMlp && !tree_too) {
                } else if (use_grid) {
                    // MortonTraceVertexT::Commit (OPX7UtilsMorton.h:550-585) ->
                    // MortonQuadTreeWrapperT::Record: leaf of the cell's building quadtree
                    if (isfinite(irr) && irr > 0.0f) {
                        const uint32_t cell = T.v_cell[vi];
                        k_s = ((unsigned long long)cell << (2 * T.mqt.level)) + T.v_slot[vi];
                        v_s = to_fx(irr, T.mqt.fx, T.mqt.status);
                    }
                } else {
                    const uint32_t dt = T.v_cell[vi];  // stree_lookup of the vertex, from k_bounce
                    k_w = dt;
                    v_w = to_fx(1.0f, T.tree.fx, T.tree.status);
                    if (isfinite(irr) && irr > 0.0f) {
                        k_s = T.v_slot[vi];
                        v_s = to_fx(irr, T.tree.fx, T.tree.status);
                    }
                }
            }
        }
        if (G == kGuideMlp && !tree_too) {
        } else if (use_grid) {
            warp_add_u64(k_s, v_s, T.mqt.leaves);
        } else {
            if (k_w != ~0ull) atomicAdd(priv_w ? s_w + k_w : T.tree.b_statw + k_w, v_w);
            if (k_s != ~0ull) atomicAdd(priv ? s_q + k_s : T.tree.b_sums + k_s, v_s);
        }
    }
    }
    if (priv_w) {
        __syncthreads();
        if (priv)
            for (uint32_t j = threadIdx.x; j < nq; j += blockDim.x)
                if (s_q[j]) atomicAdd(T.tree.b_sums + j, s_q[j]);
        for (uint32_t j = threadIdx.x; j < ndt; j += blockDim.x)
            if (s_w[j]) atomicAdd(T.tree.b_statw + j, s_w[j]);
    }
}

__global__ void k_tri_frames(const float* __restrict__ tri_v, uint32_t n, TriFrame* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* tv = tri_v + 9 * size_t(i);
        out[i] = make_tri_frame(f3(tv[0], tv[1], tv[2]), f3(tv[3], tv[4], tv[5]), f3(tv[6], tv[7], tv[8]));
    }
}

__global__ void k_seed_init(uint32_t* seeds, uint32_t n, uint32_t seed) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        seeds[p] = pcg1d(pcg1d(p) ^ (seed * 0x9E3779B9u)) | 1u;
}

template <class T>
__global__ void k_image(const double* accum, uint32_t n, double inv, T* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x)
        out[i] = (T)(accum[i] * inv);
}

}  // namespace rtpg

using namespace rtpg;

struct rtpg_tracer {
    TracerDev dev{};
    rtpg_scene* scene = nullptr;
    std::vector<void*> allocs;
    // host copies for parameter updates and the adjoint
    std::vector<Material> hmats;
    std::vector<float3> hemit;
    std::vector<int32_t> light_mat;  // material of every light mesh (-1: its triangles differ)
    bool light_mat_shared = false;   // some material belongs to two light meshes
    float3* col_adj = nullptr;       // path colour of the adjoint replay
    float3* lrem = nullptr;
    int32_t* d_mat_light = nullptr;
    std::vector<const float*> tex_ptr;
    std::vector<int32_t> mat_tex;  // texture index of every material (host copy for checks)
    std::vector<uint2> tex_wh;
    const float** d_tex = nullptr;
    uint2* d_tex_wh = nullptr;
    uint32_t seed = 1;
    bool timing = false;
    double t_ms[3] = {0, 0, 0};  // raygen, bounce, finish
    uint64_t t_launch[3] = {0, 0, 0};
    cudaEvent_t ev[8] = {};
    uint64_t samples = 0;
    uint64_t paths = 0;
    struct Cached {
        cudaGraphExec_t exec;
        TracerDev dev;  // a captured wave bakes in every kernel argument
    };
    std::map<uint32_t, Cached> graphs;  // keyed by flags; the guide views are compared on use
    template <class T>
    int alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RTPG_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(q);
        *p = static_cast<T*>(q);
        return RTPG_OK;
    }
    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
    }
    ~rtpg_tracer() {
        drop_graphs();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (void* p : allocs) cudaFree(p);
    }
};

// The kernels of a wave are dependent launches: each may be scheduled while its predecessor
// drains and waits for it in-kernel (grid_dependency_wait), which hides the launch gaps of
// the bounce chain.  Launch errors surface at graph instantiation or the next checked call.
// One CTA per 128 queue entries of a full queue: the block scheduler hands the SMs new CTAs as
// others finish, which balances a bounce's tail better than a resident grid striding over the
// queue (measured 4% faster on the Cornell render); CTAs past the queue's end return at once.
static int bounce_grid(const TracerDev& T) { return (int)((T.npath + kTB - 1) / kTB); }
static void launch_bounce(const TracerDev& T, int g, cudaStream_t st, uint32_t b) {
    if (guide_of(T.flags) == kGuideMlp) {
        if (b == 0) (void)launch_dependent(k_hit, g, kTB, 0, st, T, b);
        if (T.flags & RTPG_TRACE_FLAG_BUILD) (void)launch_dependent(k_mlp_lobes, kSMs * 4, kMlpThreads, kSmemEval, st, T, b);
        (void)launch_dependent(k_bounce<kGuideMlp>, g, kTB, 0, st, T, b);
        return;
    }
    switch (guide_of(T.flags)) {
        case kGuideTree: (void)launch_dependent(k_bounce<kGuideTree>, g, kTB, 0, st, T, b); break;
        case kGuideGrid: (void)launch_dependent(k_bounce<kGuideGrid>, g, kTB, 0, st, T, b); break;
        default: (void)launch_dependent(k_bounce<kGuideNone>, g, kTB, 0, st, T, b); break;
    }
}
// accumulation, then (recording waves of a guide) the commit of the trace vertices: two CTAs
// of kCommitThreads per SM, each walking every vertex row over its share of the paths
static void launch_finish(const TracerDev& T, int g, cudaStream_t st) {
    (void)launch_dependent(k_finish, g, kTB, 0, st, T);
    if (T.flags & RTPG_TRACE_FLAG_FINAL) return;
    const int gc = kSMs * 2;
    switch (guide_of(T.flags)) {
        case kGuideTree: (void)launch_dependent(k_commit<kGuideTree>, gc, kCommitThreads, 0, st, T); break;
        case kGuideGrid: (void)launch_dependent(k_commit<kGuideGrid>, gc, kCommitThreads, 0, st, T); break;
        case kGuideMlp: (void)launch_dependent(k_commit<kGuideMlp>, gc, kCommitThreads, 0, st, T); break;
        default: break;
    }
}

// One wave with CUDA events around every kernel group; synchronises and accumulates the
// per-group device time (used to measure the kernels, outside the graph-replayed path).
static int timed_wave(rtpg_tracer* h, cudaStream_t st) {
    TracerDev& T = h->dev;
    const int g = kSMs * 8;
    for (auto& e : h->ev)
        if (!e) RTPG_CUDA(cudaEventCreate(&e));
    cudaEventRecord(h->ev[0], st);
    k_raygen<<<g, kTB, 0, st>>>(T);
    cudaEventRecord(h->ev[1], st);
    RTPG_CUDA(cudaEventSynchronize(h->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    h->t_ms[0] += ms;
    h->t_launch[0] += 1;
    for (uint32_t b = 0; b < T.max_depth; ++b) {
        cudaEventRecord(h->ev[2], st);
        launch_bounce(T, bounce_grid(T), st, b);
        cudaEventRecord(h->ev[3], st);
        RTPG_CUDA(cudaEventSynchronize(h->ev[3]));
        cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]);
        h->t_ms[1] += ms;
        h->t_launch[1] += 1;
    }
    cudaEventRecord(h->ev[4], st);
    launch_finish(T, g, st);
    cudaEventRecord(h->ev[5], st);
    RTPG_CUDA(cudaEventSynchronize(h->ev[5]));
    cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
    h->t_ms[2] += ms;
    h->t_launch[2] += 1;
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

static void launch_wave(rtpg_tracer* h, cudaStream_t st) {
    TracerDev& T = h->dev;
    const int g = kSMs * 8;
    (void)launch_dependent(k_raygen, g, kTB, 0, st, T);
    for (uint32_t b = 0; b < T.max_depth; ++b) launch_bounce(T, bounce_grid(T), st, b);
    launch_finish(T, g, st);
}

extern "C" {

int rtpg_tracer_create(rtpg_scene* scene, const float* tri_vertices, const uint32_t* tri_material, const float* tri_uv,
                       const rtpg_material* host_materials, uint32_t num_materials, const uint32_t* light_tris,
                       const uint32_t* host_light_mesh_first, const uint32_t* host_light_mesh_count,
                       uint32_t num_light_meshes, const rtpg_camera* host_camera, const rtpg_tracer_desc* host_desc,
                       rtpg_tracer** out) {
    if (!scene || !tri_vertices || !tri_material || !host_materials || !num_materials || !host_camera || !host_desc || !out)
        return fail(RTPG_EINVAL, "rtpg_tracer_create: null argument");
    if (num_light_meshes && (!light_tris || !host_light_mesh_first || !host_light_mesh_count))
        return fail(RTPG_EINVAL, "rtpg_tracer_create: light arrays missing");
    const rtpg_tracer_desc& D = *host_desc;
    if (!D.width || !D.height || D.max_depth < 1 || D.max_depth > 64)
        return fail(RTPG_EINVAL, "rtpg_tracer_create: bad image size or max_depth");
    auto* h = new (std::nothrow) rtpg_tracer();
    if (!h) return fail(RTPG_ENOMEM, "rtpg_tracer_create: out of host memory");
    h->scene = scene;
    TracerDev& T = h->dev;
    T.scene = scene_device_view(scene);
    T.nflat = 0;
    if (T.scene.flat && T.scene.ntris <= kFlatTris) {
        // the scene's triangles (scene order) into the kernel parameters
        const cudaError_t e = cudaMemcpy(T.ftri, T.scene.flat, sizeof(BvhTri) * T.scene.ntris, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete h;
            return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
        }
        T.nflat = T.scene.ntris;
    }
    T.tri_v = tri_vertices;
    T.tri_mat = tri_material;
    T.tri_uv = tri_uv;
    T.width = D.width;
    T.height = D.height;
    T.npath = D.width * D.height;
    T.max_depth = D.max_depth;
    T.num_candidates = D.num_candidates ? D.num_candidates : 32;
    T.bg = make_float3(D.background[0], D.background[1], D.background[2]);
    const rtpg_camera& c = *host_camera;
    T.eye = make_float3(c.eye[0], c.eye[1], c.eye[2]);
    T.cu = make_float3(c.u[0], c.u[1], c.u[2]);
    T.cv = make_float3(c.v[0], c.v[1], c.v[2]);
    T.cw = make_float3(c.w[0], c.w[1], c.w[2]);
    h->seed = D.seed ? D.seed : 1;
    const size_t P = T.npath;
    Material* mats = nullptr;
    uint2* lmesh = nullptr;
    float3* lemit = nullptr;
    int r;
    if ((r = h->alloc(&mats, num_materials)) || (r = h->alloc(&lmesh, std::max(num_light_meshes, 1u))) ||
        (r = h->alloc(&lemit, std::max(num_light_meshes, 1u))) || (r = h->alloc(&T.org, P)) ||
        (r = h->alloc(&T.dir, P)) || (r = h->alloc(&T.thr, P)) || (r = h->alloc(&T.col, P)) ||
        (r = h->alloc(&T.rng, P)) || (r = h->alloc(&T.depth, P)) ||
        (r = h->alloc(&T.hflags, P)) || (r = h->alloc(&T.queue[0], P)) ||
        (r = h->alloc(&T.queue[1], P)) || (r = h->alloc(&T.qcount, 3)) ||
        (r = h->alloc(&T.v_dir, P * kTV)) || (r = h->alloc(&T.v_thr, P * kTV)) || (r = h->alloc(&T.b_rad, P * std::max<uint32_t>(D.max_depth, 1))) ||
        (r = h->alloc(&T.v_wopdf, P * kTV)) ||
        (r = h->alloc(&T.v_cos, P * kTV)) || (r = h->alloc(&T.v_flags, P * kTV)) || (r = h->alloc(&T.v_cell, P * kTV)) || (r = h->alloc(&T.v_slot, P * kTV)) || (r = h->alloc(&T.seeds, P)) ||
        (r = h->alloc(&T.accum, 3 * P)) || (r = h->alloc(&T.status, 1)) || (r = h->alloc(&T.counters, 2)) || (r = h->alloc(&h->d_tex, 64)) ||
        (r = h->alloc(&h->d_tex_wh, 64))) {
        delete h;
        return r;
    }
    std::vector<Material> hm(num_materials);
    std::vector<float3> he(std::max(num_light_meshes, 1u));
    for (uint32_t i = 0; i < num_materials; ++i) {
        const rtpg_material& s = host_materials[i];
        Material& m = hm[i];
        m.diffuse = make_float3(s.diffuse[0], s.diffuse[1], s.diffuse[2]);
        m.specular = make_float3(s.specular[0], s.specular[1], s.specular[2]);
        m.emission = make_float3(s.emission[0], s.emission[1], s.emission[2]);
        m.shininess = s.shininess;
        m.ref_index = s.ref_index;
        m.type = s.type;
        m.tex = s.diffuse_texture;
        m.pad[0] = m.pad[1] = m.pad[2] = 0;
    }
    std::vector<uint2> hl(std::max(num_light_meshes, 1u), make_uint2(0, 1));
    for (uint32_t i = 0; i < num_light_meshes; ++i) {
        hl[i] = make_uint2(host_light_mesh_first[i], host_light_mesh_count[i]);
        if (!host_light_mesh_count[i]) {
            delete h;
            return fail(RTPG_EINVAL, "rtpg_tracer_create: empty light mesh %u", i);
        }
        he[i] = make_float3(host_desc->light_emission ? host_desc->light_emission[3 * i] : 0.f,
                            host_desc->light_emission ? host_desc->light_emission[3 * i + 1] : 0.f,
                            host_desc->light_emission ? host_desc->light_emission[3 * i + 2] : 0.f);
    }
    cudaError_t e;
    if ((e = cudaMemcpy(mats, hm.data(), sizeof(Material) * num_materials, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(lmesh, hl.data(), sizeof(uint2) * hl.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(lemit, he.data(), sizeof(float3) * he.size(), cudaMemcpyHostToDevice))) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
    }
    T.mats = mats;
    T.num_materials = num_materials;
    for (uint32_t i = 0; i < num_materials; ++i) h->mat_tex.push_back(host_materials[i].diffuse_texture);
    T.light_mesh = lmesh;
    T.light_emit = lemit;
    T.light_tris = light_tris;
    T.light_count = num_light_meshes;
    // light mesh <-> emissive material, for emitter parameters and their gradients
    h->hmats = hm;
    h->hemit = he;
    {
        std::vector<int32_t> ml(num_materials, -1);
        h->light_mat.assign(num_light_meshes, -1);
        uint32_t nlt = 0;
        for (uint32_t i = 0; i < num_light_meshes; ++i) nlt = std::max(nlt, hl[i].x + hl[i].y);
        std::vector<uint32_t> lt(nlt), tm;
        if (nlt && (e = cudaMemcpy(lt.data(), light_tris, 4ull * nlt, cudaMemcpyDeviceToHost))) {
            delete h;
            return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
        }
        const uint32_t nt = T.scene.ntris;
        tm.resize(nt);
        if (nlt && (e = cudaMemcpy(tm.data(), tri_material, 4ull * nt, cudaMemcpyDeviceToHost))) {
            delete h;
            return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
        }
        for (uint32_t i = 0; i < num_light_meshes; ++i) {
            int32_t mat = -1;
            for (uint32_t k = 0; k < hl[i].y; ++k) {
                const uint32_t t = lt[hl[i].x + k];
                const int32_t mk = t < nt ? (int32_t)std::min(tm[t], num_materials - 1) : -1;
                mat = (k == 0) ? mk : (mat == mk ? mat : -1);
            }
            h->light_mat[i] = mat;
            if (mat >= 0) {
                if (ml[mat] >= 0 && ml[mat] != (int32_t)i) h->light_mat_shared = true;
                ml[mat] = (int32_t)i;
            }
        }
        if (h->light_mat_shared) std::fill(ml.begin(), ml.end(), -1);
        if ((r = h->alloc(&h->d_mat_light, num_materials)) || (r = h->alloc(&h->col_adj, P)) ||
            (r = h->alloc(&h->lrem, P))) {
            delete h;
            return r;
        }
        if ((e = cudaMemcpy(h->d_mat_light, ml.data(), 4ull * num_materials, cudaMemcpyHostToDevice))) {
            delete h;
            return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
        }
        T.mat_light = h->d_mat_light;
        T.adj_tex = -1;
    }
    T.tex = h->d_tex;
    T.tex_wh = h->d_tex_wh;
    {
        TriFrame* fr = nullptr;
        if ((r = h->alloc(&fr, std::max(T.scene.ntris, 1u)))) {
            delete h;
            return r;
        }
        k_tri_frames<<<grid_for(T.scene.ntris, 256, 8), 256>>>(tri_vertices, T.scene.ntris, fr);
        if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(nullptr)) != cudaSuccess) {
            delete h;
            return fail(RTPG_ECUDA, "rtpg_tracer_create: %s", cudaGetErrorString(e));
        }
        T.tri_frame = fr;
    }
    *out = h;
    return rtpg_tracer_clear(h, nullptr);
}

int rtpg_tracer_destroy(rtpg_tracer* h) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_destroy: null handle");
    delete h;
    return RTPG_OK;
}

int rtpg_tracer_set_texture(rtpg_tracer* h, uint32_t index, uint32_t width, uint32_t height, const float* rgb) {
    if (!h || !rgb || !width || !height || index >= 64) return fail(RTPG_EINVAL, "rtpg_tracer_set_texture: bad arguments");
    if (h->tex_ptr.size() <= index) {
        h->tex_ptr.resize(index + 1, nullptr);
        h->tex_wh.resize(index + 1, make_uint2(0, 0));
    }
    h->tex_ptr[index] = rgb;
    h->tex_wh[index] = make_uint2(width, height);
    RTPG_CUDA(cudaMemcpy(h->d_tex, h->tex_ptr.data(), sizeof(float*) * h->tex_ptr.size(), cudaMemcpyHostToDevice));
    RTPG_CUDA(cudaMemcpy(h->d_tex_wh, h->tex_wh.data(), sizeof(uint2) * h->tex_wh.size(), cudaMemcpyHostToDevice));
    return RTPG_OK;
}

// Zero the accumulation and reseed every pixel's Xorshift32 stream from `seed` (the
// application reseeds from the host: RTLibExtOPX7TestApplication.cpp:2293-2299).
int rtpg_tracer_clear(rtpg_tracer* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_clear: null handle");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemsetAsync(h->dev.accum, 0, sizeof(double) * 3 * h->dev.npath, st));
    RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, 4, st));
    RTPG_CUDA(cudaMemsetAsync(h->dev.counters, 0, 16, st));
    k_seed_init<<<grid_for(h->dev.npath, 256, 4), 256, 0, st>>>(h->dev.seeds, h->dev.npath, h->seed);
    RTPG_LAUNCH_CHECK();
    h->samples = 0;
    return RTPG_OK;
}

int rtpg_tracer_set_seed(rtpg_tracer* h, uint32_t seed) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_set_seed: null handle");
    h->seed = seed ? seed : 1;
    return RTPG_OK;
}

static int check_render(rtpg_tracer* h, uint32_t flags, const char* fn) {
    if ((flags & RTPG_TRACE_FLAG_RIS) && !(flags & RTPG_TRACE_FLAG_NEE))
        return fail(RTPG_EINVAL, "%s: RIS requires NEE", fn);
    if ((flags & RTPG_TRACE_FLAG_USE_TREE) && (flags & RTPG_TRACE_FLAG_USE_GRID))
        return fail(RTPG_EINVAL, "%s: USE_TREE and USE_GRID are exclusive", fn);
    for (int32_t t : h->mat_tex)
        if (t >= 0 && (size_t(t) >= h->tex_ptr.size() || !h->tex_ptr[t]))
            return fail(RTPG_EINVAL, "%s: material texture %d was never set", fn, t);
    if (h->dev.scene.ntris == 0) return fail(RTPG_EINVAL, "%s: empty scene", fn);
    return RTPG_OK;
}

// `spp` waves with the flags and guide views already in h->dev.  A captured wave bakes in
// the kernel arguments, so it is reused only for the same flags and identical guide views
// (the same device arrays).
static int render_waves(rtpg_tracer* h, uint32_t spp, uint32_t flags, cudaStream_t st) {
    h->dev.flags = flags;
    if (h->timing) {
        for (uint32_t s = 0; s < spp; ++s) {
            int r = timed_wave(h, st);
            if (r) return r;
        }
        h->samples += spp;
        h->paths += uint64_t(spp) * h->dev.npath;
        return RTPG_OK;
    }
    auto it = h->graphs.find(flags);
    cudaGraphExec_t exec = nullptr;
    if (it != h->graphs.end() && memcmp(&it->second.dev, &h->dev, sizeof(TracerDev)) == 0) {
        exec = it->second.exec;
    } else {
        if (it != h->graphs.end()) {
            cudaGraphExecDestroy(it->second.exec);
            h->graphs.erase(it);
        }
        cudaStream_t cs;
        RTPG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            launch_wave(h, cs);
            e = cudaStreamEndCapture(cs, &g);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return fail(RTPG_ECUDA, "rtpg_tracer_render: graph capture failed: %s", cudaGetErrorString(e));
        h->graphs[flags] = {exec, h->dev};
    }
    for (uint32_t s = 0; s < spp; ++s) RTPG_CUDA(cudaGraphLaunch(exec, st));
    h->samples += spp;
    h->paths += uint64_t(spp) * h->dev.npath;
    return RTPG_OK;
}

// One launch of `spp` samples per pixel with the given RTPG_TRACE_FLAG_* (PARAM_FLAG_*,
// SimpleKernel.h:145-158).  tree may be NULL when RTPG_TRACE_FLAG_USE_TREE is not set.
int rtpg_tracer_render(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_sdtree* tree, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_render: null handle");
    if ((flags & RTPG_TRACE_FLAG_USE_TREE) && !tree) return fail(RTPG_EINVAL, "rtpg_tracer_render: USE_TREE without a tree");
    if (flags & (RTPG_TRACE_FLAG_USE_GRID | RTPG_TRACE_FLAG_LOCATE))
        return fail(RTPG_EINVAL, "rtpg_tracer_render: grid flags need rtpg_tracer_render_grid");
    int r = check_render(h, flags, "rtpg_tracer_render");
    if (r) return r;
    memset(&h->dev.grid, 0, sizeof(HashGridDev));
    memset(&h->dev.mqt, 0, sizeof(MqtDev));
    memset(&h->dev.ml, 0, sizeof(MlpView));
    if (tree) h->dev.tree = sdtree_device_view(tree);
    else memset(&h->dev.tree, 0, sizeof(SDTreeDev));
    return render_waves(h, spp, flags, as_stream(stream));
}

// One launch guided by the hash grid and its Morton quadtrees (the HT* tracers of
// SimpleGuide2.cu).
int rtpg_tracer_render_grid(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_hashgrid* grid, rtpg_mqt* mqt,
                            void* stream) {
    if (!h || !grid || !mqt) return fail(RTPG_EINVAL, "rtpg_tracer_render_grid: null argument");
    if (!(flags & RTPG_TRACE_FLAG_USE_GRID)) return fail(RTPG_EINVAL, "rtpg_tracer_render_grid: USE_GRID not set");
    int r = check_render(h, flags, "rtpg_tracer_render_grid");
    if (r) return r;
    const HashGridDev g = hashgrid_device_view(grid);
    const MqtDev q = mqt_device_view(mqt);
    if (q.ncells < g.nslots)
        return fail(RTPG_EINVAL, "rtpg_tracer_render_grid: %u quadtrees for %u grid slots", q.ncells, g.nslots);
    memset(&h->dev.tree, 0, sizeof(SDTreeDev));
    memset(&h->dev.ml, 0, sizeof(MlpView));
    h->dev.grid = g;
    h->dev.mqt = q;
    return render_waves(h, spp, flags, as_stream(stream));
}

// One launch guided by the learned mixture (no counterpart in RTLib): every bounce runs the
// closest-hit queries, the network on the tensor cores for the hit points (with BUILD), then
// shading; unless FINAL, committed trace vertices become training records of the guide, each
// kept with probability record_keep.  With a fallback SD-tree the guide density is
// mlp_share * network + (1 - mlp_share) * SD-tree, and the vertices are committed to the tree
// as well.
int rtpg_tracer_render_mlp(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_mlp* mlp, rtpg_sdtree* fallback,
                           float fraction, float mlp_share, float record_keep, void* stream) {
    if (!h || !mlp) return fail(RTPG_EINVAL, "rtpg_tracer_render_mlp: null argument");
    if (fallback && !(mlp_share >= 0.0f && mlp_share <= 1.0f))
        return fail(RTPG_EINVAL, "rtpg_tracer_render_mlp: mlp_share outside [0, 1]");
    if (!(flags & RTPG_TRACE_FLAG_USE_MLP) || (flags & (RTPG_TRACE_FLAG_USE_TREE | RTPG_TRACE_FLAG_USE_GRID)))
        return fail(RTPG_EINVAL, "rtpg_tracer_render_mlp: flags must hold USE_MLP and no other guide");
    if (!(fraction >= 0.0f && fraction <= 1.0f)) return fail(RTPG_EINVAL, "rtpg_tracer_render_mlp: fraction outside [0, 1]");
    int r = check_render(h, flags, "rtpg_tracer_render_mlp");
    if (r) return r;
    TracerDev& T = h->dev;
    if (!T.hit_prim) {
        const size_t P = T.npath;
        if ((r = h->alloc(&T.hit_prim, P)) || (r = h->alloc(&T.hit_tuv, P)) || (r = h->alloc(&T.lobes, P * 40)) ||
            (r = h->alloc(&T.v_nrm, P * kTV)) || (r = h->alloc(&T.v_wo, P * kTV)) || (r = h->alloc(&T.v_pos, P * kTV)))
            return r;
        RTPG_CUDA(cudaFuncSetAttribute(k_mlp_lobes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemEval));
    }
    if (fallback) T.tree = sdtree_device_view(fallback);
    else memset(&T.tree, 0, sizeof(SDTreeDev));
    memset(&T.grid, 0, sizeof(HashGridDev));
    memset(&T.mqt, 0, sizeof(MqtDev));
    T.ml = mlp_view(mlp);
    T.mlp_fraction = fraction;
    T.mlp_keep = record_keep;
    T.mlp_share = fallback ? mlp_share : 1.0f;
    return render_waves(h, spp, flags, as_stream(stream));
}

// Mean radiance per pixel (accumulation / samples), RGB float, row-major, y = 0 first.
int rtpg_tracer_image(rtpg_tracer* h, float* out_rgb, void* stream) {
    if (!h || !out_rgb) return fail(RTPG_EINVAL, "rtpg_tracer_image: null argument");
    const double inv = h->samples ? 1.0 / (double)h->samples : 0.0;
    k_image<<<grid_for(3ull * h->dev.npath, 256, 4), 256, 0, as_stream(stream)>>>(h->dev.accum, h->dev.npath, inv, out_rgb);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// Mean radiance per pixel in FP64 (accumulation / samples).
int rtpg_tracer_image_f64(rtpg_tracer* h, double* out_rgb, void* stream) {
    if (!h || !out_rgb) return fail(RTPG_EINVAL, "rtpg_tracer_image_f64: null argument");
    const double inv = h->samples ? 1.0 / (double)h->samples : 0.0;
    k_image<<<grid_for(3ull * h->dev.npath, 256, 4), 256, 0, as_stream(stream)>>>(h->dev.accum, h->dev.npath, inv, out_rgb);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// Device pointer to the FP64 accumulation buffer (3 doubles per pixel) and the sample count.
int rtpg_tracer_accumulation(rtpg_tracer* h, const double** dev_accum, uint64_t* host_samples) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_accumulation: null handle");
    if (dev_accum) *dev_accum = h->dev.accum;
    if (host_samples) *host_samples = h->samples;
    return RTPG_OK;
}

// Guided rendering driven by the pass controller, as TracePipeline does for the PG tracers
// (RTLibExtOPX7TestApplication.cpp:2155-2230, flags by state as in GetParams,
// RTLibExtOPX7TestApplication.h:399-424): per launch BegTrace, render samples_per_launch
// with USE_TREE (+BUILD in RECORD_AND_SAMPLE, +BUILD|FINAL in SAMPLE), EndTrace.
int rtpg_tracer_render_guided(rtpg_tracer* h, rtpg_sdtree* tree, rtpg_controller* ctrl, uint32_t base_flags,
                              uint32_t samples_per_launch, uint32_t max_launches, void* stream) {
    if (!h || !tree || !ctrl) return fail(RTPG_EINVAL, "rtpg_tracer_render_guided: null argument");
    int r;
    for (uint32_t k = 0; k < max_launches; ++k) {
        if ((r = rtpg_controller_begin(ctrl, stream))) return r;
        int32_t state, executing;
        uint32_t it, tmp;
        rtpg_controller_get(ctrl, &state, &it, &tmp, &executing);
        if (!executing) break;
        uint32_t flags = (base_flags & (RTPG_TRACE_FLAG_NEE | RTPG_TRACE_FLAG_RIS)) | RTPG_TRACE_FLAG_USE_TREE;
        if (state == RTPG_TRACE_RECORD_AND_SAMPLE) flags |= RTPG_TRACE_FLAG_BUILD;
        if (state == RTPG_TRACE_SAMPLE) flags |= RTPG_TRACE_FLAG_BUILD | RTPG_TRACE_FLAG_FINAL;
        if ((r = rtpg_tracer_render(h, samples_per_launch, flags, tree, stream))) return r;
        if ((r = rtpg_controller_end(ctrl, stream))) return r;
    }
    return RTPG_OK;
}

// TracePipeline for the HT* tracers (RTLibExtOPX7TestApplication.cpp:2174-2222): flags by
// the Morton controller's state, the grid's current table copied to the previous one after
// every finished pass (GetSamplePerTmp() == 0 after EndTrace).
int rtpg_tracer_render_grid_guided(rtpg_tracer* h, rtpg_hashgrid* grid, rtpg_mqt* mqt, rtpg_mqt_controller* ctrl,
                                   uint32_t base_flags, uint32_t samples_per_launch, uint32_t max_launches,
                                   void* stream) {
    if (!h || !grid || !mqt || !ctrl) return fail(RTPG_EINVAL, "rtpg_tracer_render_grid_guided: null argument");
    int r;
    for (uint32_t k = 0; k < max_launches; ++k) {
        if ((r = rtpg_mqt_controller_begin(ctrl, stream))) return r;
        int32_t state, executing;
        uint32_t it, tmp;
        rtpg_mqt_controller_get(ctrl, &state, &it, &tmp, &executing);
        if (!executing) break;
        uint32_t flags = (base_flags & (RTPG_TRACE_FLAG_NEE | RTPG_TRACE_FLAG_RIS)) | RTPG_TRACE_FLAG_USE_GRID;
        if (state == RTPG_MQT_TRACE_LOCATE) flags |= RTPG_TRACE_FLAG_LOCATE;
        if (state == RTPG_MQT_TRACE_RECORD_AND_SAMPLE) flags |= RTPG_TRACE_FLAG_BUILD;
        if (state == RTPG_MQT_TRACE_SAMPLE) flags |= RTPG_TRACE_FLAG_BUILD | RTPG_TRACE_FLAG_FINAL;
        if ((r = rtpg_tracer_render_grid(h, samples_per_launch, flags, grid, mqt, stream))) return r;
        if ((r = rtpg_mqt_controller_end(ctrl, stream))) return r;
        rtpg_mqt_controller_get(ctrl, &state, &it, &tmp, &executing);
        if (tmp == 0 && (r = rtpg_hashgrid_swap(grid, stream))) return r;
    }
    return RTPG_OK;
}

// Emitter radiances: light mesh i gets rgb[3i..3i+2] for NEE (MeshLight::emission) and as the
// emission of its material (what a ray that hits it sees).
int rtpg_tracer_set_light_emission(rtpg_tracer* h, const float* host_rgb, uint32_t num_lights) {
    if (!h || !host_rgb) return fail(RTPG_EINVAL, "rtpg_tracer_set_light_emission: null argument");
    if (num_lights != h->dev.light_count)
        return fail(RTPG_EINVAL, "rtpg_tracer_set_light_emission: %u values for %u lights", num_lights, h->dev.light_count);
    if (h->light_mat_shared)
        return fail(RTPG_EINVAL, "rtpg_tracer_set_light_emission: light meshes share an emissive material");
    for (uint32_t i = 0; i < num_lights; ++i) {
        if (h->light_mat[i] < 0)
            return fail(RTPG_EINVAL, "rtpg_tracer_set_light_emission: light mesh %u has triangles of several materials", i);
        h->hemit[i] = make_float3(host_rgb[3 * i], host_rgb[3 * i + 1], host_rgb[3 * i + 2]);
        h->hmats[h->light_mat[i]].emission = h->hemit[i];
    }
    RTPG_CUDA(cudaMemcpy(const_cast<float3*>(h->dev.light_emit), h->hemit.data(), sizeof(float3) * num_lights,
                         cudaMemcpyHostToDevice));
    RTPG_CUDA(cudaMemcpy(const_cast<Material*>(h->dev.mats), h->hmats.data(), sizeof(Material) * h->hmats.size(),
                         cudaMemcpyHostToDevice));
    return RTPG_OK;
}

__global__ void k_seed_store(TracerDev T) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < T.npath; p += gridDim.x * blockDim.x)
        T.seeds[p] = T.rng[p];
}

// Path-replay backpropagation of an image loss.  Replays the `spp` samples that
// rtpg_tracer_render(h, spp, flags) draws from the current per-pixel streams: per sample one
// primal wave gives every path's radiance, one adjoint wave runs the same path again and
// scatters gradients.  The streams advance as that render would advance them; the
// accumulation is not touched.
int rtpg_tracer_render_adjoint(rtpg_tracer* h, uint32_t spp, uint32_t flags, const float* d_image,
                               int32_t texture_index, float* grad_texture, float* grad_light_emission, void* stream) {
    if (!h || !d_image) return fail(RTPG_EINVAL, "rtpg_tracer_render_adjoint: null argument");
    if (flags & ~RTPG_TRACE_FLAG_NEE)
        return fail(RTPG_EINVAL, "rtpg_tracer_render_adjoint: only the unguided tracer with or without NEE is differentiated "
                                 "(RIS resampling weights depend on the emitter radiances)");
    if (texture_index >= 0 && (!grad_texture || size_t(texture_index) >= h->tex_ptr.size() || !h->tex_ptr[texture_index]))
        return fail(RTPG_EINVAL, "rtpg_tracer_render_adjoint: texture %d not set or no gradient buffer", texture_index);
    if (grad_light_emission && h->light_mat_shared)
        return fail(RTPG_EINVAL, "rtpg_tracer_render_adjoint: light meshes share an emissive material");
    int r = check_render(h, flags, "rtpg_tracer_render_adjoint");
    if (r) return r;
    if (!aligned4(d_image) || (grad_texture && !aligned4(grad_texture)) || (grad_light_emission && !aligned4(grad_light_emission)))
        return fail(RTPG_EINVAL, "rtpg_tracer_render_adjoint: misaligned buffer");
    cudaStream_t st = as_stream(stream);
    TracerDev A = h->dev;
    A.flags = flags;
    memset(&A.tree, 0, sizeof(SDTreeDev));
    memset(&A.grid, 0, sizeof(HashGridDev));
    memset(&A.mqt, 0, sizeof(MqtDev));
    A.adj_c = nullptr;
    TracerDev B = A;
    B.col = h->col_adj;
    B.adj_c = A.col;
    B.lrem = h->lrem;
    B.adj_dimg = d_image;
    B.adj_scale = spp ? 1.0f / (float)spp : 0.0f;
    B.adj_tex = texture_index;
    B.grad_tex = texture_index >= 0 ? grad_texture : nullptr;
    B.grad_light = grad_light_emission;
    const int g = kSMs * 8;
    for (uint32_t s = 0; s < spp; ++s) {
        k_raygen<<<g, kTB, 0, st>>>(A);
        for (uint32_t b = 0; b < A.max_depth; ++b) k_bounce<kGuideNone><<<g, kTB, 0, st>>>(A, b);
        k_raygen<<<g, kTB, 0, st>>>(B);
        for (uint32_t b = 0; b < B.max_depth; ++b) k_bounce<kAdjoint><<<g, kTB, 0, st>>>(B, b);
        k_seed_store<<<g, kTB, 0, st>>>(B);
    }
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_tracer_counters(rtpg_tracer* h, uint64_t* host_path_bounces, uint64_t* host_shadow_rays, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_counters: null handle");
    unsigned long long c[2];
    RTPG_CUDA(cudaMemcpyAsync(c, h->dev.counters, sizeof(c), cudaMemcpyDeviceToHost, as_stream(stream)));
    RTPG_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (host_path_bounces) *host_path_bounces = c[0];
    if (host_shadow_rays) *host_shadow_rays = c[1];
    return RTPG_OK;
}

// Debug view of the last wave: final bounce index of every path and the number of trace
// vertices it committed or would commit (n = min(depth, 10) when recording).
int rtpg_tracer_path_depths(rtpg_tracer* h, uint32_t* out_depth, void* stream) {
    if (!h || !out_depth) return fail(RTPG_EINVAL, "rtpg_tracer_path_depths: null argument");
    RTPG_CUDA(cudaMemcpyAsync(out_depth, h->dev.depth, sizeof(uint32_t) * h->dev.npath, cudaMemcpyDeviceToDevice,
                              as_stream(stream)));
    return RTPG_OK;
}

int rtpg_tracer_set_timing(rtpg_tracer* h, int enable) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_set_timing: null handle");
    h->timing = enable != 0;
    for (int k = 0; k < 3; ++k) {
        h->t_ms[k] = 0.0;
        h->t_launch[k] = 0;
    }
    return RTPG_OK;
}

int rtpg_tracer_timings(rtpg_tracer* h, double* host_ms, uint64_t* host_launches) {
    if (!h || !host_ms) return fail(RTPG_EINVAL, "rtpg_tracer_timings: null argument");
    for (int k = 0; k < 3; ++k) {
        host_ms[k] = h->t_ms[k];
        if (host_launches) host_launches[k] = h->t_launch[k];
    }
    return RTPG_OK;
}

int rtpg_tracer_stats(rtpg_tracer* h, uint64_t* host_samples, uint64_t* host_paths) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_tracer_stats: null handle");
    if (host_samples) *host_samples = h->samples;
    if (host_paths) *host_paths = h->paths;
    return RTPG_OK;
}

}  // extern "C"
