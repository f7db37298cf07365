"""The bench's reading of the committed ncu summaries (no GPU): the DRAM traffic
of a kernel is reported only while the hash of the code it was captured from
equals the hash of the code being built, and that hash ignores comments."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_code_only_drops_comments_and_keeps_strings():
    src = ('int a = 1;  // one\n/* block\n   comment */\nconst char* s = "// kept";\n\n'
           'asm("add.rn.f32x2 %0, %1;" : "=l"(x));  /* tail */\nchar c = \'/\';\n')
    out = bench.code_only(src)
    assert "one" not in out and "block" not in out and "tail" not in out
    assert '"// kept"' in out and "add.rn.f32x2" in out and "'/'" in out
    assert bench.code_only(src.replace("// one", "// changed comment")) == out
    assert bench.code_only(src.replace("int a = 1", "int a = 2")) != out


def test_profile_traffic_follows_the_source_hash():
    for kernel in bench.PROFILE_SOURCES:
        value, src = bench.profile_traffic(kernel, "multilayer_512x512x8")
        assert os.path.exists(os.path.join(ROOT, src["file"]))
        assert src["sources_sha"] is not None and len(src["sources_sha"]) == 16
        assert src["build_sources_sha"] == bench.kernel_sources_sha(bench.PROFILE_SOURCES[kernel])
        if src["matches_build"]:
            assert value is not None and value > 0
        else:
            assert value is None
