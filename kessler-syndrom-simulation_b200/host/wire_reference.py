"""Wires the B200 engine into a copy of the reference and builds its CLI.

This is the maintainer's side of the drop-in, done by a script: it copies the
reference's src/ tree to a temporary directory (the reference itself is never
modified), inserts there the engine behind the reference's screening and step calls,
and builds the reference's own main.cpp against libkessler_b200.so:

  src/core/collision.cpp   Screener::set_gpu / gpu / gpu_compiled / begin /
                           finish: with set_gpu(true) the screening of each
                           step runs on the engine (kessler_b200::Screener,
                           host/kessler_b200.hpp) with the reference's own
                           State / Object / Conjunction types.
  src/core/orbital.cpp     Simulation::step: every step runs on the engine
                           (kessler_b200::step_objects).

Every edit is an insertion guarded by KESSLER_HAS_B200 right after a line of
the reference found by exact match (each anchor must occur exactly once, or
the script stops), so the same sources still build without the engine. The
result is <package>/_wired/kessler_sim: the reference CLI, unchanged in its
options and output files, whose --gpu switch selects the engine.

    python wire_reference.py [--reference DIR] [--out DIR]

DIR defaults to the KESSLER_REFERENCE environment variable, else
/root/reference. No file of the reference is copied into this repository.
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)

# (file, anchor line, text inserted after it). Anchors are whole lines of the
# reference, matched after stripping trailing whitespace.
EDITS = [
    ("core/collision.cpp", '#include "collision.hpp"',
     '#ifdef KESSLER_HAS_B200\n#include "kessler_b200.hpp"\n#endif'),
    ("core/collision.cpp", "struct Screener::Impl {",
     "#ifdef KESSLER_HAS_B200\n"
     "    kessler_b200::Screener b200;  // the B200 engine behind set_gpu(true)\n"
     "#endif"),
    ("core/collision.cpp", "bool Screener::gpu_compiled() {",
     "#ifdef KESSLER_HAS_B200\n    return true;\n#endif"),
    ("core/collision.cpp", "bool Screener::set_gpu(bool on, std::string* message) {",
     "#ifdef KESSLER_HAS_B200\n"
     "    impl_->launched = false;\n"
     "    return impl_->b200.set_gpu(on, message);  // no CPU fallback: false + message if no device\n"
     "#endif"),
    ("core/collision.cpp", "bool Screener::gpu() const {",
     "#ifdef KESSLER_HAS_B200\n    return impl_->b200.gpu();\n#endif"),
    ("core/collision.cpp",
     "void Screener::begin(const std::vector<State>& before, const std::vector<Object>& objects, double dt) {",
     "#ifdef KESSLER_HAS_B200\n"
     "    // The engine screens the whole step in finish(); nothing to launch ahead.\n"
     "    if (impl_->b200.gpu()) {\n"
     "        impl_->launched = false;\n"
     "        return;\n"
     "    }\n"
     "#endif"),
    ("core/orbital.cpp", '#include "orbital.hpp"',
     '#ifdef KESSLER_HAS_B200\n#include "kessler_b200.hpp"\n#endif'),
    ("core/orbital.cpp", "void Simulation::step() {",
     "#ifdef KESSLER_HAS_B200\n"
     "    // One device round trip per call: states and alive flags in, RK4 step\n"
     "    // (re-entries killed) on the GPU, states back; t advanced as below.\n"
     "    static kessler_b200::Context* b200_ctx = new kessler_b200::Context(0);\n"
     "    t = kessler_b200::step_objects(*b200_ctx, objects, epoch_jd, t, dt, 1);\n"
     "    return;\n"
     "#endif"),
]

# Screener::finish: its signature spans lines; the anchor is its first line,
# and the insertion goes after the line that ends the signature.
FINISH_FIRST = "std::vector<Conjunction> Screener::finish(const std::vector<State>& before,"
FINISH_BODY = """#ifdef KESSLER_HAS_B200
    if (impl_->b200.gpu()) {
        kessler_b200::ScreeningConfig& c = impl_->b200.config();
        c.threshold_km = cfg_.threshold_km;
        c.radius_scale = cfg_.radius_scale;
        c.min_encounter_speed_km_s = cfg_.min_encounter_speed_km_s;
        ks_step_stats st{};
        std::vector<Conjunction> out = impl_->b200.screen<Conjunction>(before, after, t0, dt, &st);  // (t, i, j) order
        if (stats) {
            *stats = ScreeningStats{};
            stats->candidate_pairs = st.candidate_pairs;
            stats->refined_pairs = st.refined_pairs;
            stats->co_orbiting = st.co_orbiting;
            stats->cell_km = st.cell_km;
            stats->max_cell_objects = st.max_cell_objects;
            stats->max_cell_pairs = static_cast<long long>(st.max_cell_objects) * (st.max_cell_objects - 1) / 2;
            stats->threads = 0;
            stats->gpu = true;
        }
        return out;
    }
#endif"""


def reference_tree(arg):
    return arg or os.environ.get("KESSLER_REFERENCE", "/root/reference")


def apply_edits(src):
    """Applies EDITS to the copy under `src` (the copy of the reference's src/)."""
    for rel, anchor, text in EDITS:
        path = os.path.join(src, rel)
        lines = open(path).read().split("\n")
        hits = [k for k, ln in enumerate(lines) if ln.rstrip() == anchor]
        if len(hits) != 1:
            raise SystemExit(f"{rel}: anchor found {len(hits)} times, expected once: {anchor!r}")
        lines[hits[0] + 1:hits[0] + 1] = text.split("\n")
        open(path, "w").write("\n".join(lines))
    # Screener::finish: insert after the line that closes its signature.
    path = os.path.join(src, "core/collision.cpp")
    lines = open(path).read().split("\n")
    hits = [k for k, ln in enumerate(lines) if ln.rstrip() == FINISH_FIRST]
    if len(hits) != 1:
        raise SystemExit(f"core/collision.cpp: Screener::finish found {len(hits)} times")
    k = hits[0]
    while not lines[k].rstrip().endswith("{"):
        k += 1
        if k - hits[0] > 4:
            raise SystemExit("core/collision.cpp: end of Screener::finish's signature not found")
    lines[k + 1:k + 1] = FINISH_BODY.split("\n")
    open(path, "w").write("\n".join(lines))


def build(reference, out_dir, cxx="g++"):
    src_ref = os.path.join(reference, "src")
    if not os.path.isdir(src_ref):
        raise SystemExit(f"reference tree not found: {src_ref}")
    lib = os.path.join(PKG, "libkessler_b200.so")
    if not os.path.exists(lib):
        raise SystemExit("build the engine first (make -C kessler-syndrom-simulation_b200)")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "kessler_sim")
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "src")
        shutil.copytree(src_ref, src)
        apply_edits(src)
        core = [os.path.join(src, "core", f) for f in ("orbital.cpp", "collision.cpp", "breakup.cpp", "threads.cpp")]
        # The reference's own flags for its CPU build (-O3, OpenMP, no FMA
        # contraction), plus the engine's headers and library.
        cmd = [cxx, "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-DKESSLER_HAS_B200",
               "-I" + src, "-I" + os.path.join(ROOT, "include"), "-I" + HERE] + core + \
              [os.path.join(src, "main.cpp"), "-L" + PKG, "-lkessler_b200",
               "-Wl,-rpath,$ORIGIN/" + os.path.relpath(PKG, out_dir), "-o", exe]
        subprocess.run(cmd, check=True)
    return exe


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--out", default=os.path.join(PKG, "_wired"))
    a = ap.parse_args()
    exe = build(reference_tree(a.reference), a.out)
    print(exe)
    return 0


if __name__ == "__main__":
    sys.exit(main())
