"""The build module must import in a tree where nothing is compiled yet,
and the product must fail loudly there instead of falling back."""
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_build_module_imports_before_build(tmp_path):
    src = os.path.join(ROOT, "tomocam_b200")
    dst = tmp_path / "tomocam_b200"
    dst.mkdir()
    for f in os.listdir(src):
        if f.endswith(".py"):
            shutil.copy(os.path.join(src, f), dst / f)
    code = (
        "import tomocam_b200, tomocam_b200.build as b\n"
        "assert callable(b.build)\n"
        "try:\n"
        "    tomocam_b200.radon\n"
        "except ImportError as e:\n"
        "    assert 'not built' in str(e)\n"
        "else:\n"
        "    raise SystemExit('radon resolved without the compiled module')\n"
    )
    env = dict(os.environ, PYTHONPATH=str(tmp_path))
    r = subprocess.run([sys.executable, "-c", code], cwd=tmp_path, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
