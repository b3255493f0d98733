"""The C++ adapter (rypath_b200/adapter) compiled against rypath's own headers.

The adapter takes the place of src/metal_render_stub.cpp in rypath's backend library: it
defines build_metal_renderer, MetalRenderScene and the frame-session entry points of
src/metal_render.hpp:14-95 and src/frame_session.hpp over include/rypath_cuda.h.  Compiling it
against a rypath checkout's headers and linking it to librypath_cuda.so shows that the C ABI
binds the reference's interface as its code declares it: every reference symbol the stub
defines is defined here with the same C++ signature, and every rp_cuda_* symbol it calls is
exported by the library.  The Film conversion (film_fold) is checked against rypath's FilmPixel.

The adapter is built by rypath_b200/adapter/Makefile, from __graft_entry__.build() when a rypath
checkout is present, or here when RYPATH_REFERENCE names one.
"""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "rypath_b200", "adapter")
BUILD = os.path.join(ADAPTER, "_build")
LIB = os.path.join(ROOT, "rypath_b200", "librypath_cuda.so")

# what src/metal_render_stub.cpp defines, as demangled by nm
REFERENCE_SYMBOLS = [
    "rypath::build_metal_renderer(rypath::RenderScene const&, std::filesystem::__cxx11::path const&)",
    "rypath::build_metal_renderer(rypath::RenderScene const&, std::filesystem::__cxx11::path const&, "
    "rypath::RenderTimings*)",
    "rypath::build_metal_renderer(rypath::RenderScene const&, std::filesystem::__cxx11::path const&, "
    "rypath::RenderBuildOptions, rypath::RenderTimings*)",
    "rypath::MetalRenderScene::sample(rypath::RenderRequest const&)",
    "rypath::MetalRenderScene::sample(rypath::RenderRequest const&, rypath::RenderTimings&)",
    "rypath::MetalRenderScene::~MetalRenderScene()",
    "rypath::MetalRenderScene::MetalRenderScene(rypath::MetalRenderScene&&)",
    "rypath::MetalRenderScene::operator=(rypath::MetalRenderScene&&)",
    "rypath::probe_shading_normal(std::vector<rypath::shading_normal_probe::Query, "
    "std::allocator<rypath::shading_normal_probe::Query> > const&, std::filesystem::__cxx11::path const&)",
    "rypath::build_frame_session(rypath::RenderScene const&, rypath::FrameConfig const&, "
    "std::filesystem::__cxx11::path const&)",
    "rypath::FrameSession::submit(rypath::FrameRequest const&)",
    "rypath::Frame::poll() const",
    "rypath::Frame::wait() const",
    "rypath::Frame::capture() const",
    "rypath::cuda_backend::FilmRenderer::build(rypath::RenderScene const&, std::__cxx11::basic_string<char, "
    "std::char_traits<char>, std::allocator<char> >&)",
]


def built():
    lib = os.path.join(BUILD, "libcuda_render.so")
    if not os.path.exists(lib):
        ref = os.environ.get("RYPATH_REFERENCE")
        if not ref or not os.path.isdir(os.path.join(ref, "src")):
            pytest.skip("adapter not built and RYPATH_REFERENCE names no rypath checkout")
        subprocess.run(["make", "-s", "-C", ADAPTER, f"REF={ref}"], check=True)
    return lib


def symbols(path, *flags):
    """Demangled dynamic symbol names of `path` (nm lines: [address] type name)."""
    import re

    out = subprocess.run(["nm", "-C", "-D", *flags, path], capture_output=True, text=True, check=True).stdout
    names = set()
    for line in out.splitlines():
        m = re.match(r"^\s*(?:[0-9a-fA-F]+\s+)?[A-Za-z]\s+(.*\S)\s*$", line)
        if m:
            names.add(m.group(1))
    return names


def test_adapter_defines_the_reference_interface():
    lib = built()
    defined = symbols(lib, "--defined-only")
    missing = [s for s in REFERENCE_SYMBOLS if s not in defined]
    assert not missing, missing


def test_adapter_calls_only_exported_entry_points():
    lib = built()
    needed = subprocess.run(["readelf", "-d", lib], capture_output=True, text=True, check=True).stdout
    assert "[librypath_cuda.so]" in needed
    calls = {s for s in symbols(lib, "--undefined-only") if s.startswith("rp_cuda_")}
    exported = {s for s in symbols(LIB, "--defined-only") if s.startswith("rp_cuda_")}
    assert {"rp_cuda_scene_create", "rp_cuda_sample", "rp_cuda_sample_scalar", "rp_cuda_render_film",
            "rp_cuda_frame_session_create", "rp_cuda_frame_submit", "rp_cuda_frame_capture"} <= calls
    assert calls <= exported, calls - exported


def test_film_fold_matches_rypath_film_pixel():
    built()
    run = subprocess.run([os.path.join(BUILD, "film_fold_check")], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
