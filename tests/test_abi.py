"""The C ABI library: loads, exports every declared entry point, and fails
loudly (a status code, no fallback) when no GPU is present.  CPU only."""
import ctypes
import os
import re

import pytest

import beedrill_b200 as bd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(bd_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(bd.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) > 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_status_strings_and_version():
    L = bd.lib()
    for code in range(0, -11, -1):
        assert L.bd_status_string(code)
    assert b"sm_100a" in L.bd_version()


def test_no_gpu_means_error_not_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bd.BeedrillError) as ei:
        bd.Graph.rmat(8)
    assert ei.value.status == -9  # BD_ERR_NODEV


def test_algorithm_names_cover_reference_cli():
    # hybrid_bfs_main.cc:228-245 accepts these four
    for name in ("remote_writes", "migrating_threads", "remote_writes_hybrid", "beamer_hybrid"):
        assert name in bd.ALGORITHMS
    with pytest.raises(ValueError):
        bd.HybridBFS.__init__(object.__new__(bd.HybridBFS), None, alg="bogus")


def test_invalid_arguments_rejected_without_device():
    L = bd.lib()
    h = ctypes.c_void_p()
    assert L.bd_graph_rmat(0, 16, 0.57, 0.19, 0.19, 0.05, 0, 0, ctypes.byref(h)) == -1
    assert L.bd_graph_rmat(10, 16, 0.57, 0.19, 0.19, 0.05, 0, 7, ctypes.byref(h)) == -1
    assert L.bd_bfs_create(None, None, ctypes.byref(h)) == -1
    assert L.bd_components_create(None, ctypes.byref(h)) == -1
    assert L.bd_components_run(None, None) == -1
    ok, bad = ctypes.c_int32(), ctypes.c_int64()
    assert L.bd_graph_check_parents(None, 0, None, ctypes.byref(ok), ctypes.byref(bad)) == -1
    assert L.bd_graph_check_components(None, None, ctypes.byref(ok), ctypes.byref(bad)) == -1


def test_cpp_facade_reads_the_trained_policies(tmp_path):
    """The C++ facade's JSON reader (used by the CLI's --algorithm learned)
    gets the same numbers the Python trainer wrote."""
    import json
    import subprocess
    src = tmp_path / "load.cc"
    src.write_text(
        '#include "beedrill/hybrid_bfs.hpp"\n'
        'int main(int argc, char **argv) {\n'
        '  beedrill::policy p = beedrill::load_policy(argv[1]);\n'
        '  double s = 0; for (float v : p.params) s += v;\n'
        '  printf("%zu %zu %zu %zu %.6g %.9g %.9g\\n", p.params.size(), p.mean.size(), p.lo.size(),\n'
        '         p.hi.size(), p.margin, s, p.inv_std[3]);\n'
        '  try { beedrill::load_policy(argv[2]); } catch (const beedrill::error &e) {\n'
        '    printf("%d\\n", (int)e.status); }\n'
        '  return 0; }\n')
    exe = tmp_path / "load"
    lib_dir = os.path.dirname(bd.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", lib_dir, "-lbeedrill_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    bad = tmp_path / "bad.json"
    bad.write_text('{"params": [1, 2, 3], "mean": [0]}')
    for name in ("learned_policy.json", "learned_policy_batched.json"):
        path = os.path.join(ROOT, "beedrill_b200", "policy", name)
        if not os.path.exists(path):
            continue
        out = subprocess.run([str(exe), path, str(bad)], check=True, stdout=subprocess.PIPE,
                             text=True).stdout.split()
        d = json.load(open(path))
        assert out[:4] == ["1410", "8", "8", "8"]
        margin = float(out[4])  # +inf: a policy that leaves every step to the rule
        assert margin == d["margin"] or abs(margin - d["margin"]) <= 1e-6 * max(1.0, abs(d["margin"]))
        assert abs(float(out[5]) - sum(d["params"])) <= 1e-3 * max(1.0, sum(abs(v) for v in d["params"]))
        assert abs(float(out[6]) - d["inv_std"][3]) <= 1e-6 * abs(d["inv_std"][3])
        assert out[7] == "-3"  # BD_ERR_FORMAT


def test_cpp_facade_reads_the_tuning_file(tmp_path):
    """The C++ facade's reader of the autotuner's file (used by the CLI)
    picks the same entry, with the same values, as the Python binding."""
    import subprocess
    src = tmp_path / "tune.cc"
    src.write_text(
        '#include "beedrill/hybrid_bfs.hpp"\n'
        'int main(int argc, char **argv) {\n'
        '  beedrill::tuning t = beedrill::load_tuning(argv[1], atol(argv[2]));\n'
        '  bd_bfs_opts o; memset(&o, 0, sizeof o); t.apply(&o);\n'
        '  bd_msbfs_opts m; memset(&m, 0, sizeof m); m.alpha = 4; t.apply(&m);\n'
        '  printf("%d %d %d %d %d %d %lld %d %d %d %d %d %d\\n", o.block_size, o.large_degree,\n'
        '         o.chunk_edges, o.bu_prefix, o.bu_words, o.bu_sparse_words, (long long)m.alpha,\n'
        '         m.block_size, m.large_degree, m.chunk_edges, m.pull_prefix, m.heavy_degree,\n'
        '         m.heavy_chunk);\n'
        '  return 0; }\n')
    exe = tmp_path / "tune"
    lib_dir = os.path.dirname(bd.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", lib_dir, "-lbeedrill_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    path = os.path.join(ROOT, "beedrill_b200", "tuning", "b200.json")
    if not os.path.exists(path):
        pytest.skip("no tuning file committed")
    for n in (1 << 16, 1 << 20, 1 << 21, 1 << 23, 1 << 24, 1 << 26):
        out = [int(x) for x in subprocess.run([str(exe), path, str(n)], check=True,
                                               stdout=subprocess.PIPE, text=True).stdout.split()]
        s, b = bd.tuned_options("single", n), bd.tuned_options("batched", n)
        want = [s.get(k, 0) for k in ("block_size", "large_degree", "chunk_edges", "bu_prefix",
                                      "bu_words", "bu_sparse_words")] + \
               [b.get("alpha", 4)] + [b.get(k, 0) for k in ("block_size", "large_degree", "chunk_edges",
                                                             "pull_prefix", "heavy_degree", "heavy_chunk")]
        assert out == want, (n, out, want)


def test_clis_fail_loudly_without_a_device():
    """Both CLIs exit non-zero with the library's no-device status: there is
    no CPU path behind them."""
    import subprocess
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    for name in ("hybrid_bfs", "components"):
        cli = os.path.join(ROOT, "beedrill_b200", "bin", name)
        if not os.path.exists(cli):
            pytest.skip("CLIs not built")
        out = subprocess.run([cli, "--rmat_scale", "8"], stdout=subprocess.PIPE,
                             stderr=subprocess.STDOUT, text=True, timeout=120)
        assert out.returncode != 0, (name, out.stdout)
        assert "device" in out.stdout.lower(), (name, out.stdout)
        assert "Found" not in out.stdout and "Traversed" not in out.stdout


def test_cpp_facade_dump_text_equals_the_reference(tmp_path):
    """components::dump text (the CLI's --dump_results) from the facade's
    printer equals, byte for byte, what the reference's own components CLI
    printed for the same labels (tests/golden/ref_components.npz)."""
    import subprocess
    import numpy as np
    src = tmp_path / "dump.cc"
    src.write_text(
        '#include "beedrill/hybrid_bfs.hpp"\n'
        'int main(int argc, char **argv) {\n'
        '  FILE *f = fopen(argv[1], "rb"); int64_t n = 0;\n'
        '  if (!f || fread(&n, 8, 1, f) != 1) return 2;\n'
        '  std::vector<int64_t> c(n);\n'
        '  if (fread(c.data(), 8, n, f) != (size_t)n) return 2;\n'
        '  fclose(f); beedrill::detail::print_components(c, stdout); return 0; }\n')
    exe = tmp_path / "dump"
    lib_dir = os.path.dirname(bd.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", lib_dir, "-lbeedrill_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    ref = np.load(os.path.join(ROOT, "tests", "golden", "ref_components.npz"))
    for name in ("scale10", "rmat12_ef2", "grid48", "tail_isolated", "tail_path"):
        labels = ref[f"{name}.labels"]
        path = tmp_path / f"{name}.bin"
        path.write_bytes(np.int64(len(labels)).tobytes() + labels.astype(np.int64).tobytes())
        out = subprocess.run([str(exe), str(path)], check=True, stdout=subprocess.PIPE).stdout
        assert out == bytes(ref[f"{name}.dump"]), name


def test_cpp_facade_print_tree_equals_the_reference(tmp_path):
    """hybrid_bfs::print_tree text from the facade's printer equals, byte for
    byte, the reference's own print_tree() on its 8 scale-10 trees
    (tests/golden/ref_check.npz)."""
    import subprocess
    import numpy as np
    src = tmp_path / "tree.cc"
    src.write_text(
        '#include "beedrill/hybrid_bfs.hpp"\n'
        'int main(int argc, char **argv) {\n'
        '  FILE *f = fopen(argv[1], "rb"); int64_t n = 0;\n'
        '  if (!f || fread(&n, 8, 1, f) != 1) return 2;\n'
        '  std::vector<int64_t> p(n);\n'
        '  if (fread(p.data(), 8, n, f) != (size_t)n) return 2;\n'
        '  fclose(f); beedrill::detail::print_tree(p, stdout); return 0; }\n')
    exe = tmp_path / "tree"
    lib_dir = os.path.dirname(bd.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", lib_dir, "-lbeedrill_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    golden = os.path.join(ROOT, "tests", "golden")
    trees = np.load(os.path.join(golden, "ref_scale10.npz"))["beamer_hybrid.parent"]
    d = np.load(os.path.join(golden, "ref_check.npz"))
    text, off = bytes(d["tree_text"]), d["tree_offsets"]
    assert len(off) == len(trees) + 1
    for i, parent in enumerate(trees):
        path = tmp_path / f"p{i}.bin"
        path.write_bytes(np.int64(len(parent)).tobytes() + parent.astype(np.int64).tobytes())
        out = subprocess.run([str(exe), str(path)], check=True, stdout=subprocess.PIPE).stdout
        assert out == text[off[i]:off[i + 1]], i


def test_python_print_tree_text_equals_the_reference():
    import numpy as np
    golden = os.path.join(ROOT, "tests", "golden")
    trees = np.load(os.path.join(golden, "ref_scale10.npz"))["beamer_hybrid.parent"]
    d = np.load(os.path.join(golden, "ref_check.npz"))
    text, off = bytes(d["tree_text"]), d["tree_offsets"]
    for i, parent in enumerate(trees):
        assert bd.format_tree(parent).encode() == text[off[i]:off[i + 1]], i


def test_format_tree_stops_on_a_cycle():
    """A planted parent cycle (0 -> 1 -> 2 -> 1) ends its lines with a cycle
    mark instead of climbing forever, as the reference would."""
    import numpy as np
    text = bd.format_tree(np.array([1, 2, 1, -1], np.int64))
    lines = text.splitlines()
    assert len(lines) == 3
    assert all(line.endswith(" <- (cycle)") for line in lines)
    assert lines[0].startswith("   0 <-    1 <-    2 <-    1")
