// Reference oracle driver: runs RTLib's OWN guiding code on the host.
//
// Test infrastructure only (a checker, never the product).  This file is this project's
// code; it includes the reference headers staged by stage_ref.py and drives them the way
// RTLib's application does, minus the CUDA buffers:
//   * SD-tree (OPX7UtilsPathGuiding.h): the host RTSTreeT / RTDTreeWrapperT objects own the
//     trees; for record / sample / pdf they are flattened into the device-side structs
//     (STreeNodeT, DTreeWrapperT, DTreeNodeT) exactly as RTSTreeWrapperT::Upload does
//     (OPX7UtilsPathGuiding.h:1353-1564) but into host vectors, and the device routines run
//     on the host (RTLIB_DEVICE expands to nothing, atomics fall back to '+=',
//     OPX7UtilsPathGuiding.h:98-104).  After recording, the building nodes are copied back as
//     RTSTreeWrapperT::Download does (:1565-1615).
//   * Hash grid (OPX7UtilsGrid.h): DoubleBufferedHashGrid3T over host checksum arrays,
//     sequential insertion in index order.
//   * Morton quadtree (OPX7UtilsMorton.h): MortonQuadTreeT<6> on host weight arrays; the
//     pyramid reduction of mortonBuildKernel (OPX7UtilsMortonBuild.cu:2-16) is restated with
//     exact integer powers of four instead of __powf.
#include <cmath>
#include <cstring>
#include <cstdint>
#include <iostream>
#include <limits>
#include <bitset>
#include <vector>
namespace std { using ::powf; using ::expf; using ::logf; using ::sinf; using ::cosf; using ::tanf; using ::sqrtf; using ::fabsf; }
using std::isfinite;
using std::isnan;
#include <cuda_runtime.h>
#include <RTLib/Ext/OPX7/Utils/OPX7UtilsPathGuiding.h>
#include <RTLib/Ext/OPX7/Utils/OPX7UtilsMorton.h>
#include <RTLib/Ext/OPX7/Utils/OPX7UtilsGrid.h>

using namespace RTLib::Ext::OPX7::Utils;
namespace M = RTLib::Ext::CUDA::Math;

// Same template arguments as the reference build (OPX7/CMakeLists.txt:90-92).
using RSTree = RTSTreeT<69, 24>;
using RDTree = RTDTreeT<24>;
using RDTreeWrapper = RTDTreeWrapperT<24>;
using DTreeWrapper = DTreeWrapperT<24>;
using DTree = DTreeT<24>;
using DTreeNode = DTreeNodeT<24>;
using STreeNode = STreeNodeT<69, 24>;
using STree = STreeT<69, 24>;

struct RefSDTree {
    RSTree cpu;
    // flattened device-style view
    std::vector<STreeNode> sNodes;
    std::vector<DTreeWrapper> wrappers;
    std::vector<DTreeNode> bNodes, sampNodes;
    std::vector<size_t> leafOfWrapper;
    STree view{};
    RefSDTree(float3 mn, float3 mx) : cpu(mn, mx) {}

    // RTSTreeWrapperT::Upload (OPX7UtilsPathGuiding.h:1353-1517) into host vectors.
    void flatten() {
        const size_t n = cpu.GetNumNodes();
        size_t nW = 0, nB = 0, nS = 0;
        for (size_t i = 0; i < n; ++i) {
            if (cpu.Node(i).isLeaf) {
                ++nW;
                nB += cpu.Node(i).dTree.building.GetNumNodes();
                nS += cpu.Node(i).dTree.sampling.GetNumNodes();
            }
        }
        sNodes.assign(n, STreeNode{});
        wrappers.assign(nW, DTreeWrapper{});
        bNodes.assign(nB, DTreeNode{});
        sampNodes.assign(nS, DTreeNode{});
        leafOfWrapper.assign(nW, 0);
        size_t w = 0, ob = 0, os = 0;
        for (size_t i = 0; i < n; ++i) {
            auto& node = cpu.Node(i);
            sNodes[i] = node.GetGpuHandle();
            if (node.isLeaf) {
                sNodes[i].dTree = wrappers.data() + w;
                wrappers[w].building = node.dTree.building.GetGpuHandle();
                wrappers[w].building.nodes = bNodes.data() + ob;
                for (size_t j = 0; j < node.dTree.building.GetNumNodes(); ++j)
                    bNodes[ob + j] = node.dTree.building.Node(j);
                ob += node.dTree.building.GetNumNodes();
                wrappers[w].sampling = node.dTree.sampling.GetGpuHandle();
                wrappers[w].sampling.nodes = sampNodes.data() + os;
                for (size_t j = 0; j < node.dTree.sampling.GetNumNodes(); ++j)
                    sampNodes[os + j] = node.dTree.sampling.Node(j);
                os += node.dTree.sampling.GetNumNodes();
                leafOfWrapper[w] = i;
                ++w;
            } else {
                sNodes[i].dTree = nullptr;
            }
        }
        view.nodes = sNodes.data();
        view.aabbMin = cpu.GetAabbMin();
        view.aabbMax = cpu.GetAabbMax();
        view.fraction = 0.0f;
    }
    // RTSTreeWrapperT::Download (OPX7UtilsPathGuiding.h:1565-1615).
    void unflatten() {
        for (size_t w = 0; w < wrappers.size(); ++w) {
            auto& dt = cpu.Node(leafOfWrapper[w]).dTree.building;
            dt.SetGpuHandle(wrappers[w].building);
            const DTreeNode* src = wrappers[w].building.nodes;
            for (size_t j = 0; j < dt.GetNumNodes(); ++j) dt.Node(j) = src[j];
        }
    }
};

// ---------------------------------------------------------------------------------------
// canonical export: pre-order streams, identical format to the product's export
//   stree_mask[k]   : 1 interior / 0 leaf, STree pre-order (child 0 before child 1)
//   per leaf (pre-order): 4 scalars {building statW, sampling sum, sampling area,
//                         sampling statW} and the node count of the selected DTree
//   dtree stream     : per DTree node in pre-order (quadrant 0..3): child mask (bit i set
//                      when quadrant i has a child) and 4 float sums
// ---------------------------------------------------------------------------------------
static void export_dtree(const std::vector<DTreeNode>& nodes, size_t idx, std::vector<uint8_t>& masks,
                         std::vector<float>& sums) {
    const DTreeNode& nd = nodes[idx];
    uint8_t m = 0;
    for (int i = 0; i < 4; ++i)
        if (!nd.IsLeaf(i)) m |= uint8_t(1u << i);
    masks.push_back(m);
    for (int i = 0; i < 4; ++i) sums.push_back(nd.GetSum(i));
    for (int i = 0; i < 4; ++i)
        if (!nd.IsLeaf(i)) export_dtree(nodes, nd.GetChild(i), masks, sums);
}

struct ExportBuf {
    std::vector<uint8_t> smask;
    std::vector<float> scalars;   // 4 per leaf
    std::vector<int64_t> counts;  // dtree node count per leaf
    std::vector<uint8_t> dmask;
    std::vector<float> dsums;
};

static void export_stree(RefSDTree* t, size_t idx, int sampling, ExportBuf& e) {
    auto& node = t->cpu.Node(idx);
    e.smask.push_back(node.isLeaf ? 0 : 1);
    if (node.isLeaf) {
        auto& w = node.dTree;
        e.scalars.push_back(w.building.GetStatisticalWeight());
        e.scalars.push_back(w.sampling.GetSum());
        e.scalars.push_back(w.sampling.GetArea());
        e.scalars.push_back(w.sampling.GetStatisticalWeight());
        auto& dt = sampling ? w.sampling : w.building;
        std::vector<DTreeNode> nodes(dt.GetNumNodes());
        for (size_t j = 0; j < nodes.size(); ++j) nodes[j] = dt.Node(j);
        size_t before = e.dmask.size();
        export_dtree(nodes, 0, e.dmask, e.dsums);
        e.counts.push_back(int64_t(e.dmask.size() - before));
        return;
    }
    export_stree(t, node.children[0], sampling, e);
    export_stree(t, node.children[1], sampling, e);
}

static thread_local ExportBuf g_export;

extern "C" {

void* ref_sdtree_new(const float* mn, const float* mx) {
    return new RefSDTree(make_float3(mn[0], mn[1], mn[2]), make_float3(mx[0], mx[1], mx[2]));
}
void ref_sdtree_free(void* h) { delete static_cast<RefSDTree*>(h); }

// Device record path run on the host: STreeT::GetDTreeWrapper (OPX7UtilsPathGuiding.h:639-648)
// then DTreeWrapperT::Record (:514-520) with the canonical direction given directly
// (uv != null) or computed by dir_to_canonical from dir_xyz (uv == null).
void ref_sdtree_record(void* h, int64_t n, const float* pos, const float* uv, const float* dir_xyz,
                       const float* radiance, const float* wo_pdf, const float* stat_w,
                       const uint8_t* is_delta) {
    auto* t = static_cast<RefSDTree*>(h);
    t->flatten();
    for (int64_t i = 0; i < n; ++i) {
        float3 p = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        DTreeWrapper* w = t->view.GetDTreeWrapper(p);
        DTreeRecord rec{};
        rec.radiance = radiance[i];
        rec.woPdf = wo_pdf ? wo_pdf[i] : 1.0f;
        rec.statisticalWeight = stat_w ? stat_w[i] : 1.0f;
        rec.isDelta = is_delta ? (is_delta[i] != 0) : false;
        if (uv) {
            if (!rec.isDelta) {
                float irradiance = rec.radiance / rec.woPdf;
                w->building.RecordIrradiance<DirectionalFilterNearest>(make_float2(uv[2 * i], uv[2 * i + 1]),
                                                                        irradiance, rec.statisticalWeight);
            }
        } else {
            rec.direction = make_float3(dir_xyz[3 * i], dir_xyz[3 * i + 1], dir_xyz[3 * i + 2]);
            w->Record<DirectionalFilterNearest>(rec);
        }
    }
    t->unflatten();
}

// RTSTreeWrapperT::Build (OPX7UtilsPathGuiding.h:1657-1663): every leaf RTDTreeWrapperT::Build.
void ref_sdtree_build(void* h) {
    auto* t = static_cast<RefSDTree*>(h);
    for (size_t i = 0; i < t->cpu.GetNumNodes(); ++i)
        if (t->cpu.Node(i).isLeaf) t->cpu.Node(i).dTree.Build();
}

// RTSTreeWrapperT::Reset body (OPX7UtilsPathGuiding.h:1645-1656) with the threshold given:
// RTSTreeT::Refine(th, maxMB), then RTDTreeWrapperT::Reset(maxDepth, subdivTh) on every leaf.
void ref_sdtree_refine(void* h, uint64_t spatial_th, int max_mb, int max_dtree_depth, float subdiv_th) {
    auto* t = static_cast<RefSDTree*>(h);
    t->cpu.Refine(size_t(spatial_th), max_mb);
    for (size_t i = 0; i < t->cpu.GetNumNodes(); ++i)
        if (t->cpu.Node(i).isLeaf) t->cpu.Node(i).dTree.Reset(max_dtree_depth, subdiv_th);
}

// The threshold formula of RTSTreeWrapperT::Reset (OPX7UtilsPathGuiding.h:1649).
uint64_t ref_sdtree_threshold(int iter, int spp) {
    size_t th = std::sqrt(std::pow(2.0, iter) * spp / 4.0f) * 4000;
    return th;
}

int64_t ref_sdtree_num_stree_nodes(void* h) { return (int64_t)static_cast<RefSDTree*>(h)->cpu.GetNumNodes(); }

// Export; returns sizes in out_sizes[5] = {smask, leaves, dnodes, -, -}.
void ref_sdtree_export(void* h, int sampling, int64_t* out_sizes) {
    auto* t = static_cast<RefSDTree*>(h);
    g_export = ExportBuf{};
    export_stree(t, 0, sampling, g_export);
    out_sizes[0] = (int64_t)g_export.smask.size();
    out_sizes[1] = (int64_t)g_export.counts.size();
    out_sizes[2] = (int64_t)g_export.dmask.size();
}
void ref_sdtree_export_copy(uint8_t* smask, float* scalars, int64_t* counts, uint8_t* dmask, float* dsums) {
    std::memcpy(smask, g_export.smask.data(), g_export.smask.size());
    std::memcpy(scalars, g_export.scalars.data(), g_export.scalars.size() * sizeof(float));
    std::memcpy(counts, g_export.counts.data(), g_export.counts.size() * sizeof(int64_t));
    std::memcpy(dmask, g_export.dmask.data(), g_export.dmask.size());
    std::memcpy(dsums, g_export.dsums.data(), g_export.dsums.size() * sizeof(float));
}

// Guided sample + pdf as the closest-hit program does (SimpleGuide.cu:322-369):
//   leaf = STreeT::GetDTreeWrapper(pos); uv = DTreeT::Sample(rng) (clamped canonical);
//   pdf_uv = DTreeT::Pdf(uv); dir = normalize(canonical_to_dir(uv)); pdf_dir = DTreeWrapperT::Pdf(dir).
// One Xorshift32 per query seeded with seeds[i].  threads > 1 splits the queries across
// std::thread workers (embarrassingly parallel; used for the host-core baseline).
}
#include <thread>
static void sample_range(RefSDTree* t, int64_t a, int64_t b, const float* pos, const uint32_t* seeds, float* out_uv,
                         float* out_pdf_uv, float* out_dir, float* out_pdf_dir) {
    for (int64_t i = a; i < b; ++i) {
        float3 p = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        const DTreeWrapper* w = t->view.GetDTreeWrapper(p);
        M::Xorshift32 rng(seeds[i]);
        float2 uv = w->sampling.Sample(rng);
        if (out_uv) { out_uv[2 * i] = uv.x; out_uv[2 * i + 1] = uv.y; }
        if (out_pdf_uv) out_pdf_uv[i] = w->sampling.Pdf(uv);
        if (out_dir || out_pdf_dir) {
            float3 d = M::normalize(M::canonical_to_dir(uv));
            if (out_dir) { out_dir[3 * i] = d.x; out_dir[3 * i + 1] = d.y; out_dir[3 * i + 2] = d.z; }
            if (out_pdf_dir) out_pdf_dir[i] = w->Pdf(d);
        }
    }
}
extern "C" {
void ref_sdtree_sample_pdf(void* h, int64_t n, const float* pos, const uint32_t* seeds, float* out_uv,
                           float* out_pdf_uv, float* out_dir, float* out_pdf_dir, int threads) {
    auto* t = static_cast<RefSDTree*>(h);
    t->flatten();
    if (threads <= 1) {
        sample_range(t, 0, n, pos, seeds, out_uv, out_pdf_uv, out_dir, out_pdf_dir);
        return;
    }
    std::vector<std::thread> th;
    for (int k = 0; k < threads; ++k) {
        int64_t a = n * k / threads, b = n * (k + 1) / threads;
        th.emplace_back(sample_range, t, a, b, pos, seeds, out_uv, out_pdf_uv, out_dir, out_pdf_dir);
    }
    for (auto& x : th) x.join();
}

// DTreeT::Pdf at given canonical points (OPX7UtilsPathGuiding.h:485-490).
void ref_sdtree_pdf(void* h, int64_t n, const float* pos, const float* uv, float* out_pdf) {
    auto* t = static_cast<RefSDTree*>(h);
    t->flatten();
    for (int64_t i = 0; i < n; ++i) {
        float3 p = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        const DTreeWrapper* w = t->view.GetDTreeWrapper(p);
        out_pdf[i] = w->sampling.Pdf(make_float2(uv[2 * i], uv[2 * i + 1]));
    }
}

// ---------------------------------------------------------------- math / rng known answers
uint32_t ref_pcg1d(uint32_t x) { return M::pcg1d(x); }
uint32_t ref_xxhash(uint32_t x) { return M::xxhash(x); }
void ref_xorshift32_floats(uint32_t seed, int n, float* out, uint32_t* out_state) {
    M::Xorshift32 r(seed);
    for (int i = 0; i < n; ++i) out[i] = M::random_float1(r);
    *out_state = r.m_seed;
}
void ref_dir_to_canonical(int64_t n, const float* d, float* uv) {
    for (int64_t i = 0; i < n; ++i) {
        float2 c = M::dir_to_canonical(make_float3(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
        uv[2 * i] = c.x; uv[2 * i + 1] = c.y;
    }
}
void ref_canonical_to_dir(int64_t n, const float* uv, float* d) {
    for (int64_t i = 0; i < n; ++i) {
        float3 v = M::canonical_to_dir(make_float2(uv[2 * i], uv[2 * i + 1]));
        d[3 * i] = v.x; d[3 * i + 1] = v.y; d[3 * i + 2] = v.z;
    }
}

// ---------------------------------------------------------------- hash grid (OPX7UtilsGrid.h)
// DoubleBufferedHashGrid3T<32>::FindFromCur (insert, :189-216 -> GetCurCellIndex :246-277) in
// index order, and FindFromPrv (lookup, :217-227 -> GetPrvCellIndex :278-300).
static DoubleBufferedHashGrid3T<32> make_grid(const float* off, const float* size, const uint32_t* bounds,
                                              uint32_t nslots, uint32_t* prv, uint32_t* cur) {
    DoubleBufferedHashGrid3T<32> g{};
    g.aabbOffset = make_float3(off[0], off[1], off[2]);
    g.aabbSize = make_float3(size[0], size[1], size[2]);
    g.bounds = make_uint3(bounds[0], bounds[1], bounds[2]);
    g.size = nslots;
    g.prvCheckSums = prv;
    g.curCheckSums = cur;
    return g;
}
void ref_hashgrid_insert(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* bounds,
                         uint32_t nslots, uint32_t* cur_checksums, uint32_t* out_slot) {
    auto g = make_grid(off, size, bounds, nslots, nullptr, cur_checksums);
    for (int64_t i = 0; i < n; ++i)
        out_slot[i] = g.FindFromCur(make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
}
void ref_hashgrid_lookup(int64_t n, const float* pos, const float* off, const float* size, const uint32_t* bounds,
                         uint32_t nslots, uint32_t* prv_checksums, uint32_t* out_slot) {
    auto g = make_grid(off, size, bounds, nslots, prv_checksums, nullptr);
    for (int64_t i = 0; i < n; ++i)
        out_slot[i] = g.FindFromPrv(make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
}

// ---------------------------------------------------------------- Morton quadtree (OPX7UtilsMorton.h)
// MortonQuadTreeT<6>::Record (leaf only, :262-285) into weights[cell * count + ...].
void ref_mqt_record(int64_t n, uint32_t level, uint32_t count_per_cell, float* weights, const uint32_t* cell,
                    const float* uv, const float* value) {
    for (int64_t i = 0; i < n; ++i) {
        if (cell[i] == UINT32_MAX) continue;  // MortonQuadTreeWrapperT::Record, :477-484
        MortonQuadTreeT<6> t(level, weights + size_t(count_per_cell) * cell[i]);
        t.Record(make_float2(uv[2 * i], uv[2 * i + 1]), value[i]);
    }
}
// Pyramid reduction of mortonBuildKernel (OPX7UtilsMortonBuild.cu:2-16), per cell, in the
// same float accumulation order; the level offsets use exact powers of four.
void ref_mqt_build(uint32_t ncells, uint32_t level, uint32_t count_per_cell, float* weights) {
    for (uint32_t c = 0; c < ncells; ++c) {
        float* w = weights + size_t(count_per_cell) * c;
        for (uint32_t i = 0; i < level; ++i) {
            uint32_t srcOff = ((1u << (2 * (level - i))) - 1) / 3;
            uint32_t dstOff = ((1u << (2 * (level - 1 - i))) - 1) / 3;
            uint32_t cnt = 1u << (2 * (level - i));
            for (uint32_t code = 0; code < cnt; ++code) w[dstOff + (code >> 2)] += w[srcOff + code];
        }
    }
}
// MortonQuadTreeT<6>::SampleAndPdf (:286-344) and ::Pdf (:401-414).
void ref_mqt_sample_pdf(int64_t n, uint32_t level, uint32_t count_per_cell, const float* weights, const uint32_t* cell,
                        const uint32_t* seeds, float* out_uv, float* out_pdf, float* out_pdf_eval) {
    for (int64_t i = 0; i < n; ++i) {
        MortonQuadTreeT<6> t(level, const_cast<float*>(weights) + size_t(count_per_cell) * cell[i]);
        M::Xorshift32 rng(seeds[i]);
        float pdf = 0.0f;
        float2 uv = t.SampleAndPdf(pdf, rng);
        out_uv[2 * i] = uv.x; out_uv[2 * i + 1] = uv.y;
        out_pdf[i] = pdf;
        if (out_pdf_eval) out_pdf_eval[i] = t.Pdf(uv);
    }
}
uint32_t ref_morton2_code(uint32_t x, uint32_t y) { return Morton2Utils<3>::GetCodeFromPosIdx((unsigned char)x, (unsigned char)y); }

}  // extern "C"

// ---------------------------------------------------------------- integrator known answers
// RTLib's closest-hit shading (SimpleGuide.cu:287-496), its light sampling and reservoir
// (SimpleKernel.h:26-143) and its BSDF sampling helpers (SimpleGuide.cu:28-47), staged by
// stage_ref.py, run on the host.  What the OptiX launch would supply comes from here:
// textures are white (tex2D returns 1), `params` holds the flags, the light list and the
// SD-tree view, and TraceOccluded is answered by brute force over the scene's triangles.
#include <cstdio>
template <class T>
inline T tex2D(cudaTextureObject_t, float, float) { return T{}; }
template <>
inline float4 tex2D<float4>(cudaTextureObject_t, float, float) { return make_float4(1.0f, 1.0f, 1.0f, 1.0f); }
#include <rtlib_kat/ShadeTypes.h>
namespace rtlib { namespace test {
using DTreeWrapper = DTreeWrapperT<24>;
using STree = STreeT<69, 24>;
} }
struct KatHitgroup { int type; };
struct KatUserData { float3 throughPut; unsigned int depth; };
struct KatHitRecord { unsigned int seed; unsigned int flags; KatUserData userData; };
struct KatShadeOut {
    float3 position, direction, currThroughput, bsdfVal, radiance;
    float cosine, woPdf;
    unsigned int flags, seed;
};
struct KatParams {
    unsigned int flags, maxDepth, numCandidates;
    int gasHandle;
    MeshLightList lights;
    rtlib::test::STree tree;
};
static KatParams params;  // the launch parameters the staged closest-hit body reads

struct KatScene {
    std::vector<float> tri_v;      // 9 per triangle
    std::vector<uint32_t> tri_mat;
    std::vector<float> mat_f;      // 11 per material: diffuse, specular, emission, shininess, refIndex
    std::vector<int> mat_type;     // HitgroupType
    std::vector<std::vector<float3>> lv;
    std::vector<std::vector<uint3>> li;
    std::vector<std::vector<float2>> lt;
    std::vector<MeshLight> lights;
};
static KatScene g_kat;

// TraceOccluded (SimpleKernel.h:357-366): any hit in (tmin, tmax), Moller-Trumbore
static bool TraceOccluded(int, float3 o, float3 d, float tmin, float tmax) {
    const size_t nt = g_kat.tri_mat.size();
    for (size_t k = 0; k < nt; ++k) {
        const float* q = g_kat.tri_v.data() + 9 * k;
        const float3 v0 = make_float3(q[0], q[1], q[2]);
        const float3 e1 = make_float3(q[3] - q[0], q[4] - q[1], q[5] - q[2]);
        const float3 e2 = make_float3(q[6] - q[0], q[7] - q[1], q[8] - q[2]);
        const float3 pv = M::cross(d, e2);
        const float det = M::dot(e1, pv);
        if (std::fabs(det) < 1e-20f) continue;
        const float inv = 1.0f / det;
        const float3 sv = o - v0;
        const float u = M::dot(sv, pv) * inv;
        if (u < 0.0f || u > 1.0f) continue;
        const float3 qv = M::cross(sv, e1);
        const float v = M::dot(d, qv) * inv;
        if (v < 0.0f || u + v > 1.0f) continue;
        const float t = M::dot(e2, qv) * inv;
        if (t > tmin && t < tmax) return true;
    }
    return false;
}
#include <rtlib_kat/ShadeKernel.h>

extern "C" {

// The scene of the known answers.  mat_type holds rtlib_b200's material types (0 Phong,
// 1 glass, 2 NEE light, 3 light outside the NEE list), mapped here to RTLib's HitgroupType
// (SimpleKernel.h:203-210).  Every light mesh becomes a MeshLight of unshared vertices with
// the identity transform and a white emission texture.
void ref_kat_set_scene(const float* tri_v, uint32_t ntris, const uint32_t* tri_mat, const float* mat_f,
                       const int32_t* mat_type, uint32_t nmats, const uint32_t* light_tris, const uint32_t* light_first,
                       const uint32_t* light_count, const float* light_emit, uint32_t nlights) {
    g_kat = KatScene{};
    g_kat.tri_v.assign(tri_v, tri_v + 9 * size_t(ntris));
    g_kat.tri_mat.assign(tri_mat, tri_mat + ntris);
    g_kat.mat_f.assign(mat_f, mat_f + 11 * size_t(nmats));
    static const int kType[4] = {HIT_GROUP_TYPE_PHONG, HIT_GROUP_TYPE_GLASS, HIT_GROUP_TYPE_NEE_LIGHT,
                                 HIT_GROUP_TYPE_DEF_LIGHT};
    for (uint32_t i = 0; i < nmats; ++i) g_kat.mat_type.push_back(kType[mat_type[i] & 3]);
    g_kat.lv.resize(nlights);
    g_kat.li.resize(nlights);
    g_kat.lt.resize(nlights);
    for (uint32_t i = 0; i < nlights; ++i) {
        for (uint32_t k = 0; k < light_count[i]; ++k) {
            const float* q = tri_v + 9 * size_t(light_tris[light_first[i] + k]);
            for (int c = 0; c < 3; ++c) {
                g_kat.lv[i].push_back(make_float3(q[3 * c], q[3 * c + 1], q[3 * c + 2]));
                g_kat.lt[i].push_back(make_float2(0.0f, 0.0f));
            }
            g_kat.li[i].push_back(make_uint3(3 * k, 3 * k + 1, 3 * k + 2));
        }
    }
    for (uint32_t i = 0; i < nlights; ++i) {
        MeshLight l{};
        l.vertices = g_kat.lv[i].data();
        l.normals = nullptr;
        l.texCrds = g_kat.lt[i].data();
        l.indices = g_kat.li[i].data();
        l.indCount = light_count[i];
        l.emission = make_float3(light_emit[3 * i], light_emit[3 * i + 1], light_emit[3 * i + 2]);
        l.transform = M::Matrix4x4::Identity();
        l.emissionTex = 0;
        g_kat.lights.push_back(l);
    }
}

// sampleCosinePDF / samplePhongPDF (SimpleGuide.cu:28-42), random_in_unit_triangle
// (Random.h:289-296): Xorshift32 states in/out, one per case.
void ref_kat_cosine(int64_t n, const float* normal, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        M::Xorshift32 rng(state[i]);
        const float3 d = sampleCosinePDF(make_float3(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]), rng);
        out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
        state[i] = rng.m_seed;
    }
}
void ref_kat_phong(int64_t n, const float* refl, const float* shininess, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        M::Xorshift32 rng(state[i]);
        const float3 d = samplePhongPDF(make_float3(refl[3 * i], refl[3 * i + 1], refl[3 * i + 2]), shininess[i], rng);
        out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
        state[i] = rng.m_seed;
    }
}
void ref_kat_triangle(int64_t n, const float* v, uint32_t* state, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        M::Xorshift32 rng(state[i]);
        const float* q = v + 9 * i;
        const float3 p = M::random_in_unit_triangle(make_float3(q[0], q[1], q[2]), make_float3(q[3], q[4], q[5]),
                                                    make_float3(q[6], q[7], q[8]), rng);
        out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
        state[i] = rng.m_seed;
    }
}
// Reservoir<int>::Update (SimpleKernel.h:124-143) over nseq sequences of len candidates
void ref_kat_reservoir(int64_t nseq, int32_t len, const float* w, const float* rnd, int32_t* sel, float* wsum,
                       uint32_t* m) {
    for (int64_t k = 0; k < nseq; ++k) {
        Reservoir<int> r{};
        r.y = -1;
        for (int32_t i = 0; i < len; ++i) r.Update(i, w[k * len + i], rnd[k * len + i]);
        sel[k] = r.y;
        wsum[k] = r.w_sum;
        m[k] = r.m;
    }
}
// MeshLightList::Sample (SimpleKernel.h:107-122) of the scene's lights; per case 14 floats:
// direction, normal, emission, distance, invPdf, position
void ref_kat_light(int64_t n, const float* p_in, uint32_t* state, float* out) {
    MeshLightList list{(unsigned int)g_kat.lights.size(), g_kat.lights.data()};
    for (int64_t i = 0; i < n; ++i) {
        M::Xorshift32 rng(state[i]);
        const LightRecord l = list.Sample(make_float3(p_in[3 * i], p_in[3 * i + 1], p_in[3 * i + 2]), rng);
        float* o = out + 14 * i;
        o[0] = l.direction.x; o[1] = l.direction.y; o[2] = l.direction.z;
        o[3] = l.normal.x; o[4] = l.normal.y; o[5] = l.normal.z;
        o[6] = l.emission.x; o[7] = l.emission.y; o[8] = l.emission.z;
        o[9] = l.distance; o[10] = l.invPdf;
        o[11] = l.position.x; o[12] = l.position.y; o[13] = l.position.z;
        state[i] = rng.m_seed;
    }
}
// __closesthit__radiance of n vertices: the ray (org, dir), hit distance t and triangle prim,
// and the path's throughput, hit flags and depth before the vertex.  Per case 17 floats out
// (position, direction, throughput after the vertex, BSDF value, radiance added, cosine,
// woPdf) and the hit flags; states in/out.  tree: a ref_sdtree handle (USE_TREE) or NULL.
void ref_kat_shade(uint32_t flags, uint32_t max_depth, uint32_t num_candidates, void* tree, float fraction, int64_t n,
                   const float* org, const float* dir, const float* t, const uint32_t* prim, const float* thr,
                   const uint32_t* pflags, const uint32_t* depth, uint32_t* state, float* out, uint32_t* out_flags) {
    params = KatParams{};
    params.flags = flags;
    params.maxDepth = max_depth;
    params.numCandidates = num_candidates;
    params.lights = MeshLightList{(unsigned int)g_kat.lights.size(), g_kat.lights.data()};
    if (tree) {
        auto* rt = static_cast<RefSDTree*>(tree);
        rt->flatten();
        params.tree = rt->view;
        params.tree.fraction = fraction;
    }
    for (int64_t i = 0; i < n; ++i) {
        const float* q = g_kat.tri_v.data() + 9 * size_t(prim[i]);
        const float3 p0 = make_float3(q[0], q[1], q[2]), p1 = make_float3(q[3], q[4], q[5]),
                     p2 = make_float3(q[6], q[7], q[8]);
        const float3 fNormal = M::normalize(M::cross(p1 - p0, p2 - p0));  // GetTriangleFNormal, identity transform
        const float3 inDir = make_float3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        const float3 position = make_float3(org[3 * i], org[3 * i + 1], org[3 * i + 2]) + t[i] * inDir;
        const uint32_t mi = g_kat.tri_mat[prim[i]];
        const float* mf = g_kat.mat_f.data() + 11 * size_t(mi);
        KatHitgroup hg{g_kat.mat_type[mi]};
        KatHitRecord hrec{};
        hrec.seed = state[i];
        hrec.flags = pflags[i];
        hrec.userData.throughPut = make_float3(thr[3 * i], thr[3 * i + 1], thr[3 * i + 2]);
        hrec.userData.depth = depth[i];
        KatShadeOut so{};
        // white textures: SampleDiffuse / SampleSpecular / SampleEmission return the factors
        kat_closesthit(&hg, &hrec, position, inDir, fNormal, fNormal, make_float3(mf[0], mf[1], mf[2]),
                       make_float3(mf[3], mf[4], mf[5]), make_float3(mf[6], mf[7], mf[8]), mf[10], mf[9], t[i], &so);
        float* o = out + 17 * i;
        const float3* vv[5] = {&so.position, &so.direction, &so.currThroughput, &so.bsdfVal, &so.radiance};
        for (int k = 0; k < 5; ++k) { o[3 * k] = vv[k]->x; o[3 * k + 1] = vv[k]->y; o[3 * k + 2] = vv[k]->z; }
        o[15] = so.cosine;
        o[16] = so.woPdf;
        out_flags[i] = so.flags;
        state[i] = so.seed;
    }
}

}  // extern "C"
