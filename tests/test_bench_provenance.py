"""The bench's ncu traffic figure is tied to the kernel sources' code: comment edits keep a
capture matched, code edits (string literals included) do not."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_code_only_drops_comments_and_keeps_literals():
    b = bench()
    src = 'int a = 1; // one\n/* block\n comment */ int b = 2;\n\nconst char *s = "// not a comment";\n'
    out = b.code_only(src)
    assert "one" not in out and "block" not in out
    assert 'const char *s = "// not a comment";' in out
    assert out.splitlines() == ["int a = 1;", " int b = 2;", 'const char *s = "// not a comment";']
    # a comment edit leaves the code unchanged; a code edit does not
    assert b.code_only(src.replace("// one", "// the first")) == out
    assert b.code_only(src.replace("= 2", "= 3")) != out
    assert b.code_only("char c = '\\'' ; // x") == "char c = '\\'' ;"


def test_recorded_captures_name_their_summaries():
    b = bench()
    for kernel, rec in b.NCU_TRAFFIC.items():
        assert os.path.exists(os.path.join(ROOT, rec["summary"])), kernel
        if rec["bytes_per_launch"] is not None:
            assert len(rec["sources_sha"]) == 16 and rec.get("commit"), kernel
