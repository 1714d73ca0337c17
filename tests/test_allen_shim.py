"""The Allen drop-in compiles against the reference's own headers (no GPU needed).

cuda_hlt_b200/allen/VeloB200Sequence.cuh gives the VELO algorithms of Allen's sequences
(configuration/sequences/Velo.h) the shape of the ALGORITHM macro
(stream/gear/include/Handler.cuh:12-32), and cuda_hlt_b200/allen/VeloB200Visitors.cu their
SequenceVisitor specialisations (stream/sequence/include/SequenceVisitor.cuh:16-49), which call
this library's C ABI. This test compiles the visitors, and a translation unit that instantiates
Allen's scheduler and RunSequenceTuple over the unmodified Velo.h list, with nvcc and the
reference tree's include directories, as Allen's build would."""
import glob
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

REF = os.environ.get("VELO_REFERENCE_TREE", os.path.normpath(os.path.join(ROOT, os.pardir, "reference")))

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "stream", "gear")) or not shutil.which("nvcc"),
                                reason="needs the reference tree and nvcc")


def include_flags():
    dirs = []
    for top in ("cuda", "stream", "main", "checker", "x86"):
        dirs += sorted(d for d in glob.glob(os.path.join(REF, top, "**", "include"), recursive=True)
                       if os.path.isdir(d))
    dirs += [os.path.join(REF, "configuration", "sequences"), os.path.join(ROOT, "include"),
             os.path.join(ROOT, "cuda_hlt_b200", "allen")]
    return [f"-I{d}" for d in dirs]


def compile_tu(src, tmp_path):
    out = tmp_path / (os.path.basename(src) + ".o")
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "--expt-relaxed-constexpr",
           "-c", src, "-o", str(out)] + include_flags()
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


def test_visitors_compile(tmp_path):
    compile_tu(os.path.join(ROOT, "cuda_hlt_b200", "allen", "VeloB200Visitors.cu"), tmp_path)


def test_velo_sequence_instantiates_with_the_shim(tmp_path):
    obj = compile_tu(os.path.join(ROOT, "tests", "allen", "velo_sequence_check.cu"), tmp_path)
    # the visitors of every VELO algorithm of Velo.h are referenced by the instantiation
    syms = subprocess.run(["nm", "-C", str(obj)], capture_output=True, text=True).stdout
    for name in ("velo_estimate_input_size_t", "consolidate_velo_tracks_t", "copy_and_prefix_sum_single_block_velo_t",
                 "prefix_sum_velo_track_hit_number_t", "velo_search_by_triplet_t"):
        assert f"SequenceVisitor::visit<{name}>" in syms, name
