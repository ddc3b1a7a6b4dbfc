"""Stage RTLib's guiding headers for a host (g++) build of the reference oracle.

Test infrastructure only: nothing in the product imports this.

RTLib's guiding code (OPX7UtilsPathGuiding.h, OPX7UtilsMorton.h, OPX7UtilsGrid.h) is
header-only C++ that was written for MSVC/nvcc.  GCC rejects a handful of MSVC-isms, so
this script copies the two headers that need it into ``oracle/_ref/include`` (git-ignored)
and applies *mechanical* fixes that change no arithmetic:

* ``template`` disambiguators on dependent member-template calls
  (OPX7UtilsPathGuiding.h:518,592,654,716,777,801,811,865);
* the in-class explicit specialisations ``Impl<DirectionalFilter...>``
  (OPX7UtilsPathGuiding.h:415-443) and ``Impl<SpatialFilter...>`` (:792-813) become partial
  specialisations on a defaulted dummy ``int`` parameter;
* ``RTSTreeWrapper2T`` (OPX7UtilsPathGuiding.h:2167-2396), which calls members that do not
  exist and is never instantiated, and its alias (:2404) are removed;
* OPX7UtilsMorton.h:371 ``random_float1(0.0f,1.0f)(rng)`` -> ``random_float1(rng)`` and
  :394-395 ``indices[0]/[1]`` -> ``indices.x/.y`` (both inside the unused ``Sample``);
* Random.h:129-137,189-197 build ``make_floatN(random_float1(rng), random_float1(rng), ...)``,
  whose argument evaluation order C++ leaves unspecified.  The device build (nvcc's cicc)
  evaluates left to right; GCC evaluates right to left, which would swap the x/y draws.  The
  staged copy sequences the draws left to right, i.e. the device order.

Every other header (Math, Hash, VectorFunction, OPX7UtilsGrid.h) is used in place
from the reference tree through ``-I``; a lower-case ``math`` symlink fixes the include
case in Hash.h:3-4 and an upper-case ``EXT`` one that in Matrix.h:3.

For the integrator's known answers it also writes ``oracle/_ref/include/rtlib_kat/ShadeTypes.h``
and ``ShadeKernel.h`` from text cut out of RTLib's OptiX test programs, which include optix.h and so cannot be
compiled here as a whole:

* SimpleKernel.h:26-143 (LightRecord, MeshLight, MeshLightList, Reservoir) with its two
  ``#ifdef __CUDACC__`` guards removed, and the enums ParamFlag, HitgroupType and
  HitRecordFlag (SimpleKernel.h:149-158, 203-210, 281-289);
* SimpleGuide.cu:28-47 (sampleCosinePDF, samplePhongPDF, getValPhongPDF) with
  ``static __forceinline__ __device__`` -> ``static inline``;
* the body of __closesthit__radiance from the Xorshift32 it seeds to the emission rule
  (SimpleGuide.cu:306-496), unchanged, inside a function whose parameters carry the values
  the program's first lines read from OptiX (SimpleGuide.cu:288-304).

The first two items go to ShadeTypes.h, the last two to ShadeKernel.h.  The names the body
uses from the launch (``params``, ``TraceOccluded``, the hit record and hit-group data) are
supplied by ref_driver.cpp between the two includes.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the RTLib source tree: $RTLIB_REFERENCE, else a checkout named "reference" beside the repository
REF = os.environ.get("RTLIB_REFERENCE", os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, os.pardir,
                                                                       "reference")))
OUT = os.path.join(os.path.dirname(HERE), "_ref")
UTILS = "RTLib/Src/Ext/OPX7/Include/RTLib/Ext/OPX7/Utils"
CUDA_INC = "RTLib/Src/Ext/CUDA/Include"


def _sub(text, old, new, count):
    n = text.count(old)
    if n != count:
        raise SystemExit(f"stage_ref: expected {count} x {old!r}, found {n}")
    return text.replace(old, new)


def patch_pathguiding(src):
    t = src
    t = _sub(t, "building.RecordIrradiance<dFilter>(", "building.template RecordIrradiance<dFilter>(", 1)
    t = _sub(t, "top.curNode->dTree->Record<dFilter>(", "top.curNode->dTree->template Record<dFilter>(", 2)
    t = _sub(t, "nodes[0].Record<dFilter>(", "nodes[0].template Record<dFilter>(", 2)
    t = _sub(t, "v.dTree->Record<dFilter>(rec)", "v.dTree->template Record<dFilter>(rec)", 1)
    t = _sub(t, "sTree.Record<dFilter>(", "sTree.template Record<dFilter>(", 1)
    t = _sub(t, "Impl<sFilter>::Record<dFilter>(", "Impl<sFilter>::template Record<dFilter>(", 1)
    # in-class explicit specialisations -> partial specialisations
    t = _sub(t, "template<DirectionalFilter dFilter>\n\t\t\t\t\tstruct Impl;",
             "template<DirectionalFilter dFilter, int RefDummy = 0>\n\t\t\t\t\tstruct Impl;", 1)
    t = _sub(t, "template<>\n\t\t\t\t\tstruct Impl<DirectionalFilterNearest> {",
             "template<int RefDummy>\n\t\t\t\t\tstruct Impl<DirectionalFilterNearest, RefDummy> {", 1)
    t = _sub(t, "template<>\n\t\t\t\t\tstruct Impl<DirectionalFilterBox> {",
             "template<int RefDummy>\n\t\t\t\t\tstruct Impl<DirectionalFilterBox, RefDummy> {", 1)
    t = _sub(t, "template<SpatialFilter sFilter>\n\t\t\t\t\tstruct Impl;",
             "template<SpatialFilter sFilter, int RefDummy = 0>\n\t\t\t\t\tstruct Impl;", 1)
    t = _sub(t, "template<>\n\t\t\t\t\tstruct Impl<SpatialFilter::SpatialFilterNearest>",
             "template<int RefDummy>\n\t\t\t\t\tstruct Impl<SpatialFilter::SpatialFilterNearest, RefDummy>", 1)
    t = _sub(t, "template<>\n\t\t\t\t\tstruct Impl<SpatialFilter::SpatialFilterBox>",
             "template<int RefDummy>\n\t\t\t\t\tstruct Impl<SpatialFilter::SpatialFilterBox, RefDummy>", 1)
    # drop RTSTreeWrapper2T and its alias
    lines = t.split("\n")
    start = next(i for i, l in enumerate(lines) if "class  RTSTreeWrapper2T {" in l) - 1
    assert "template<" in lines[start]
    end = start + 1
    depth = 0
    seen = False
    while True:
        depth += lines[end].count("{") - lines[end].count("}")
        seen = seen or "{" in lines[end]
        if seen and depth == 0:
            break
        end += 1
    del lines[start:end + 1]
    lines = [l for l in lines if "using RTSTreeWrapper2 = RTSTreeWrapper2T" not in l]
    return "\n".join(lines)


def patch_morton(src):
    t = src
    t = _sub(t, "CUDA::Math::random_float1(0.0f, 1.0f)(rng)", "CUDA::Math::random_float1(rng)", 1)
    t = _sub(t, "auto  xPosIdx = indices[0];", "auto  xPosIdx = indices.x;", 1)
    t = _sub(t, "auto  yPosIdx = indices[1];", "auto  yPosIdx = indices.y;", 1)
    return t


def patch_random(src):
    t = src
    t = _sub(t, "return make_float2(random_float1(rng), random_float1(rng));",
             "const float a_ = random_float1(rng); const float b_ = random_float1(rng); return make_float2(a_, b_);", 2)
    t = _sub(t, "return make_float3(random_float1(rng), random_float1(rng), random_float1(rng));",
             "const float a_ = random_float1(rng); const float b_ = random_float1(rng); const float c_ = random_float1(rng); "
             "return make_float3(a_, b_, c_);", 2)
    t = _sub(t, "return make_float4(random_float1(rng), random_float1(rng), random_float1(rng), random_float1(rng));",
             "const float a_ = random_float1(rng); const float b_ = random_float1(rng); const float c_ = random_float1(rng); "
             "const float d_ = random_float1(rng); return make_float4(a_, b_, c_, d_);", 2)
    return t


TEST_CUDA = "RTLib/Src/Ext/OPX7/Test/cuda"


def _cut(text, start, end, include_end=False):
    a = text.index(start)
    b = text.index(end, a)
    return text[a:b + (len(end) if include_end else 0)]


def _enum(text, head):
    a = text.index(head)
    b = text.index("};", a)
    return text[a:b + 2]


def stage_shade(ref, out_dir):
    with open(os.path.join(ref, TEST_CUDA, "SimpleKernel.h"), encoding="latin-1") as f:
        sk = f.read()
    with open(os.path.join(ref, TEST_CUDA, "SimpleGuide.cu"), encoding="latin-1") as f:
        sg = f.read()
    lights = _cut(sk, "struct LightRecord", "struct ReservoirState")
    n_guard = lights.count("#ifdef __CUDACC__")
    if n_guard != 2 or lights.count("#endif") != 2:
        raise SystemExit("stage_ref: unexpected preprocessor guards in SimpleKernel.h")
    lights = "\n".join(l for l in lights.split("\n") if l.strip() not in ("#ifdef __CUDACC__", "#endif"))
    enums = "\n".join(_enum(sk, h) for h in ("enum   ParamFlag", "enum   HitgroupType", "enum   HitRecordFlag"))
    helpers = _cut(sg, "template<typename RNG>\nstatic __forceinline__ __device__ float3       sampleCosinePDF",
                   'extern "C" __global__ void     __raygen__default')
    if helpers.count("static __forceinline__ __device__") != 3:
        raise SystemExit("stage_ref: unexpected helper declarations in SimpleGuide.cu")
    helpers = helpers.replace("static __forceinline__ __device__", "static inline")
    prog = sg[sg.index('extern "C" __global__ void     __closesthit__radiance() {'):]
    body = _cut(prog, "    auto xor32 = RTLib::Ext::CUDA::Math::Xorshift32(hrec->seed);",
                "    hrec->SetGlobalRayOrigin(position);")
    head = ("// Staged by oracle/ref/stage_ref.py from RTLib's SimpleKernel.h and SimpleGuide.cu (see\n"
            "// that script).  Test infrastructure only; not part of the product.\n#pragma once\n")
    types = head + "#include <RTLib/Ext/CUDA/Math/Matrix.h>\n\n" + lights + "\n" + enums + "\n"
    text = (
        head + helpers + "\n"
        "// __closesthit__radiance (SimpleGuide.cu:287-496) from its Xorshift32 on; the parameters\n"
        "// are the values its first lines read through OptiX.\n"
        "static inline void kat_closesthit(const KatHitgroup* hgData, KatHitRecord* hrec, float3 position, float3 inDir,\n"
        "                                  float3 fNormal, float3 vNormal, float3 diffuse, float3 specular,\n"
        "                                  float3 emission, float refIndex, float shinness, float distance,\n"
        "                                  KatShadeOut* out) {\n"
        + body +
        "    out->position = position;\n    out->direction = direction;\n    out->currThroughput = currThroughput;\n"
        "    out->bsdfVal = bsdfVal;\n    out->radiance = radiance;\n    out->cosine = cosine;\n    out->woPdf = woPdf;\n"
        "    out->flags = currHitFlags;\n    out->seed = xor32.m_seed;\n}\n")
    kdir = os.path.join(out_dir, "include", "rtlib_kat")
    os.makedirs(kdir, exist_ok=True)
    with open(os.path.join(kdir, "ShadeTypes.h"), "w", encoding="latin-1") as f:
        f.write(types)
    with open(os.path.join(kdir, "ShadeKernel.h"), "w", encoding="latin-1") as f:
        f.write(text)


def main():
    if not os.path.isdir(REF):
        print(f"stage_ref: reference tree {REF} not present; nothing staged")
        return 1
    inc = os.path.join(OUT, "include", "RTLib", "Ext", "OPX7", "Utils")
    os.makedirs(inc, exist_ok=True)
    with open(os.path.join(REF, UTILS, "OPX7UtilsPathGuiding.h"), encoding="latin-1") as f:
        pg = patch_pathguiding(f.read())
    with open(os.path.join(inc, "OPX7UtilsPathGuiding.h"), "w", encoding="latin-1") as f:
        f.write(pg)
    with open(os.path.join(REF, UTILS, "OPX7UtilsMorton.h"), encoding="latin-1") as f:
        mo = patch_morton(f.read())
    with open(os.path.join(inc, "OPX7UtilsMorton.h"), "w", encoding="latin-1") as f:
        f.write(mo)
    mdir = os.path.join(OUT, "include", "RTLib", "Ext", "CUDA", "Math")
    os.makedirs(mdir, exist_ok=True)
    with open(os.path.join(REF, CUDA_INC, "RTLib", "Ext", "CUDA", "Math", "Random.h"), encoding="latin-1") as f:
        rnd = patch_random(f.read())
    with open(os.path.join(mdir, "Random.h"), "w", encoding="latin-1") as f:
        f.write(rnd)
    # OPX7UtilsGrid.h compiles as-is: expose it next to the patched headers via a symlink
    grid_link = os.path.join(inc, "OPX7UtilsGrid.h")
    if os.path.lexists(grid_link):
        os.remove(grid_link)
    os.symlink(os.path.join(REF, UTILS, "OPX7UtilsGrid.h"), grid_link)
    # lower-case include path used by Hash.h:3-4
    shim = os.path.join(OUT, "shim", "RTLib", "Ext", "CUDA")
    os.makedirs(shim, exist_ok=True)
    link = os.path.join(shim, "math")
    if os.path.lexists(link):
        os.remove(link)
    os.symlink(os.path.join(REF, CUDA_INC, "RTLib", "Ext", "CUDA", "Math"), link)
    # upper-case include path used by Matrix.h:3
    shim_up = os.path.join(OUT, "shim", "RTLib", "EXT", "CUDA")
    os.makedirs(shim_up, exist_ok=True)
    link = os.path.join(shim_up, "Math")
    if os.path.lexists(link):
        os.remove(link)
    os.symlink(os.path.join(REF, CUDA_INC, "RTLib", "Ext", "CUDA", "Math"), link)
    stage_shade(REF, OUT)
    print("stage_ref: staged patched headers into", OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main())
