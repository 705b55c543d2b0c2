"""The C++ exact CRT driver (oneesan_exact): path bound, checkpoint V4,
result manifest V4, strict solver-output handling and resume, checked on the
CPU with fake solver executables the way tests/test_exact_runner_e2e.py of the
reference does.  File formats are verified with Python's own json module, so a
checkpoint written here is byte-compatible with scripts/solve/exact_safety.py."""
import fcntl
import hashlib
import json
import os
import signal
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXACT = os.path.join(ROOT, "oneesan-gpu_b200", "oneesan_exact")
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "path_bound.json")))
COUNTS = {2: 12, 3: 184, 4: 8512, 5: 1262816, 6: 575780564, 7: 789360053252,
          8: 3266598486981642, 9: 41044208702632496804}  # scripts/test/golden_cpu.py:9-19

pytestmark = pytest.mark.skipif(not os.path.exists(EXACT), reason="oneesan_exact not built")

FAKE = r'''#!{py}
import os, sys
n = int(sys.argv[1]); mods = [int(x) for x in sys.argv[5:]]
exact = int(os.environ["FAKE_EXACT"]); mode = os.environ.get("FAKE_MODE", "ok")
print("diagnostic line without result markers n=" + str(n), flush=True)
for i, p in enumerate(mods):
    r = exact % p
    if mode == "wrong_n": n = n + 1
    if mode == "dup" and i == 1: p = mods[0]
    if mode == "noncanonical": print(f"n={{n}} residue=0{{r}} modulus={{p}} wall_s=0.5"); continue
    if mode == "big": r = p + 1
    if mode == "corrupt" and i == 0: r = (r + 1) % p
    if mode == "stop" and i == 1: sys.exit(3)
    if mode == "slow" and i == 1:
        import time; time.sleep(120)
    wall = "0.25"
    if mode == "walls": wall = ["1e-05", "0.1", "123456789012.5", "1e+16", "2.5e-07", "3.141592653589793", "0"][i % 7]
    print(f"backend=fake n={{n}} residue={{r}} modulus={{p}} extra=1 wall_s={{wall}}", flush=True)
'''


def fake_solver(tmp_path, name="fake_solver"):
    path = tmp_path / name
    path.write_text(FAKE.format(py=sys.executable))
    path.chmod(0o755)
    return str(path)


def run(n, work, binary, mode="ok", exact=None, extra=()):
    env = dict(os.environ, FAKE_EXACT=str(COUNTS[n] if exact is None else exact), FAKE_MODE=mode)
    return subprocess.run([EXACT, str(n), "--work-dir", str(work), "--binary", binary, *extra],
                          capture_output=True, text=True, env=env, timeout=120)


def canonical_digest(data, field):
    payload = {k: v for k, v in data.items() if k != field}
    return hashlib.sha256(json.dumps(payload, sort_keys=True, separators=(",", ":"),
                                     ensure_ascii=True).encode()).hexdigest()


def test_path_bound_matches_reference_for_every_n():
    for n in range(2, 28):
        r = subprocess.run([EXACT, str(n), "--work-dir", "/nonexistent/x", "--binary", "/bin/false"],
                           capture_output=True, text=True, timeout=60)
        line = r.stderr.splitlines()[0]
        g = GOLDEN["bounds"][str(n)]
        assert f"<={g['bound']} ({g['bits']} bits)" in line, (n, line)
        assert "strips=[" + ", ".join(map(str, g["strips"])) + "]" in line
        assert f"CRT primes={g['crt_primes']}" in line


@pytest.mark.parametrize("n", [2, 5, 9])
def test_full_run_writes_verified_result(tmp_path, n):
    solver = fake_solver(tmp_path)
    r = run(n, tmp_path / "w", solver)
    assert r.returncode == 0, r.stderr
    assert f"exact={COUNTS[n]}" in r.stdout
    text = (tmp_path / "w" / "exact.txt").read_text()
    assert f"exact={COUNTS[n]}\n" in text and f"n={n}\n" in text
    man = json.loads((tmp_path / "w" / "exact_manifest.json").read_text())
    assert man["format"] == "ONEESAN_EXACT_RESULT_V4"
    assert man["manifest_sha256"] == canonical_digest(man, "manifest_sha256")
    assert man["exact_decimal"] == str(COUNTS[n])
    assert man["exact_sha256"] == hashlib.sha256(text.encode()).hexdigest()
    assert man["path_bound_decimal"] == GOLDEN["bounds"][str(n)]["bound"]
    assert man["primes_used"] == GOLDEN["bounds"][str(n)]["crt_primes"]
    assert [c["modulus"] for c in man["congruences"]] == GOLDEN["primes"][:man["primes_used"]]
    ck_text = (tmp_path / "w" / "checkpoint.json").read_text()
    ck = json.loads(ck_text)
    assert man["checkpoint_sha256"] == hashlib.sha256(ck_text.encode()).hexdigest()
    # Byte-identical to Python's json.dumps(indent=2, sort_keys=True) plus the
    # canonical-JSON SHA-256 of exact_safety.py.
    assert ck_text == json.dumps(ck, indent=2, sort_keys=True, ensure_ascii=True) + "\n"
    assert ck["checkpoint_sha256"] == canonical_digest(ck, "checkpoint_sha256")
    assert ck["format_version"] == 4 and ck["n"] == n and ck["admission_certificate"] is None
    assert ck["solver"]["binary_sha256"] == hashlib.sha256(open(solver, "rb").read()).hexdigest()
    assert "drop-one subsets reconstruct the same integer" in r.stderr


def test_float_text_matches_python(tmp_path):
    # wall_s values that exercise every branch of Python's float repr
    r = run(18, tmp_path / "w", fake_solver(tmp_path), mode="walls", exact=7 ** 90)
    assert r.returncode == 0, r.stderr  # 7^90 (253 bits) is below the n=18 bound (282 bits)
    assert f"exact={7 ** 90}" in r.stdout
    text = (tmp_path / "w" / "checkpoint.json").read_text()
    ck = json.loads(text)
    assert text == json.dumps(ck, indent=2, sort_keys=True, ensure_ascii=True) + "\n"
    assert ck["checkpoint_sha256"] == canonical_digest(ck, "checkpoint_sha256")
    walls = sorted(v["wall_s"] for v in ck["residues"].values())
    assert 1e-05 in walls and 1e+16 in walls and 123456789012.5 in walls


def test_max_runs_then_resume(tmp_path):
    solver = fake_solver(tmp_path)
    r = run(9, tmp_path / "w", solver, extra=("--max-runs", "1"))
    assert r.returncode == 0 and not (tmp_path / "w" / "exact.txt").exists()
    ck = json.loads((tmp_path / "w" / "checkpoint.json").read_text())
    assert list(ck["residues"]) == ["4294967291"]
    r = run(9, tmp_path / "w", solver)
    assert r.returncode == 0 and f"exact={COUNTS[9]}" in r.stdout
    r = run(9, tmp_path / "w", solver)  # finished checkpoint: finalise again, no solver needed
    assert r.returncode == 0 and "batch run" not in r.stderr


def test_resume_from_checkpoint_written_by_python(tmp_path):
    # A checkpoint produced with the reference's own serialisation rules.
    solver = fake_solver(tmp_path)
    work = tmp_path / "w"
    work.mkdir()
    sha = hashlib.sha256(open(solver, "rb").read()).hexdigest()
    p = 4294967291
    payload = {"format_version": 4, "n": 9,
               "solver": {"binary_name": "fake_solver", "binary_sha256": sha, "git_commit": "unknown"},
               "admission_certificate": None,
               "residues": {str(p): {"residue": COUNTS[9] % p, "wall_s": 1.5, "log": "from python"}}}
    payload["checkpoint_sha256"] = canonical_digest(payload, "checkpoint_sha256")
    (work / "checkpoint.json").write_text(json.dumps(payload, indent=2, sort_keys=True) + "\n")
    r = run(9, work, solver)
    assert r.returncode == 0, r.stderr
    man = json.loads((work / "exact_manifest.json").read_text())
    assert man["congruences"][0]["log"] == "from python" and man["congruences"][0]["wall_s"] == 1.5


@pytest.mark.parametrize("mode,needle", [
    ("wrong_n", "returned n="), ("dup", "duplicate modulus"), ("noncanonical", "non-canonical"),
    ("big", "canonical range"), ("stop", "batch solver failed, rc=3"),
    ("corrupt", "path bound")])
def test_rejects_bad_solver_output(tmp_path, mode, needle):
    r = run(9, tmp_path / "w", fake_solver(tmp_path), mode=mode)
    assert r.returncode == 1
    assert needle in r.stderr, r.stderr
    assert not (tmp_path / "w" / "exact.txt").exists()


def test_rejects_tampered_checkpoint(tmp_path):
    solver = fake_solver(tmp_path)
    assert run(9, tmp_path / "w", solver, extra=("--max-runs", "1")).returncode == 0
    path = tmp_path / "w" / "checkpoint.json"
    ck = json.loads(path.read_text())
    ck["residues"]["4294967291"]["residue"] += 1
    path.write_text(json.dumps(ck, indent=2, sort_keys=True) + "\n")
    r = run(9, tmp_path / "w", solver)
    assert r.returncode == 1 and "integrity checksum mismatch" in r.stderr


def test_rejects_checkpoint_of_another_binary(tmp_path):
    a = fake_solver(tmp_path, "solver_a")
    assert run(9, tmp_path / "w", a, extra=("--max-runs", "1")).returncode == 0
    b = fake_solver(tmp_path, "solver_b")
    with open(b, "a") as f:
        f.write("# a different build\n")
    r = run(9, tmp_path / "w", b)
    assert r.returncode == 1 and "solver binary changed" in r.stderr


def test_rejects_duplicate_json_keys(tmp_path):
    solver = fake_solver(tmp_path)
    work = tmp_path / "w"
    work.mkdir()
    (work / "checkpoint.json").write_text('{"n": 9, "n": 9}')
    r = run(9, work, solver)
    assert r.returncode == 1 and "duplicate JSON key" in r.stderr


def test_workdir_lock(tmp_path):
    work = tmp_path / "w"
    work.mkdir()
    with open(work / ".solve.lock", "a+") as f:
        fcntl.flock(f.fileno(), fcntl.LOCK_EX | fcntl.LOCK_NB)
        r = run(9, work, fake_solver(tmp_path))
    assert r.returncode == 1 and "already in use" in r.stderr


@pytest.mark.gpu
def test_in_process_exact_count_on_gpu(tmp_path):
    env = dict(os.environ)
    r = subprocess.run([EXACT, "9", "--work-dir", str(tmp_path / "w"), "--lanes", "2"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr
    assert f"exact={COUNTS[9]}" in r.stdout
    ck = json.loads((tmp_path / "w" / "checkpoint.json").read_text())
    assert ck["solver"]["binary_name"] == "libfdp.so"


def test_solver_crash_then_resume(tmp_path):
    # The solver dies after its first residue: the driver fails, but the
    # residue it had already reported is in the durable checkpoint, and the
    # next run asks only for the rest and finishes with the exact count.
    solver = fake_solver(tmp_path)
    r = run(9, tmp_path / "w", solver, mode="stop")
    assert r.returncode == 1 and "rc=3" in r.stderr
    ck = json.loads((tmp_path / "w" / "checkpoint.json").read_text())
    assert list(ck["residues"]) == ["4294967291"]
    r = run(9, tmp_path / "w", solver)
    assert r.returncode == 0 and f"exact={COUNTS[9]}" in r.stdout
    man = json.loads((tmp_path / "w" / "exact_manifest.json").read_text())
    ck = json.loads((tmp_path / "w" / "checkpoint.json").read_text())
    assert man["exact_decimal"] == str(COUNTS[9])
    assert len(man["congruences"]) == len(ck["residues"]) == man["primes_used"]


def test_driver_killed_then_resume(tmp_path):
    # The driver (and its solver) are killed while a batch is in flight; the
    # checkpoint on disk stays a valid V4 file, the work-directory lock dies
    # with the process, and a new run resumes and finishes.
    solver = fake_solver(tmp_path)
    work = tmp_path / "w"
    env = dict(os.environ, FAKE_EXACT=str(COUNTS[9]), FAKE_MODE="slow")
    p = subprocess.Popen([EXACT, "9", "--work-dir", str(work), "--binary", solver], env=env,
                         stdout=subprocess.PIPE, stderr=subprocess.PIPE, start_new_session=True)
    ck_path = work / "checkpoint.json"
    try:
        deadline = time.time() + 60
        while time.time() < deadline:
            if ck_path.exists() and json.loads(ck_path.read_text()).get("residues"):
                break
            time.sleep(0.1)
        else:
            raise AssertionError("no checkpointed residue within 60 s")
    finally:
        os.killpg(p.pid, signal.SIGKILL)  # the process group this test started
        p.communicate(timeout=30)
    ck = json.loads(ck_path.read_text())
    assert list(ck["residues"]) == ["4294967291"]
    r = run(9, work, solver)
    assert r.returncode == 0 and f"exact={COUNTS[9]}" in r.stdout
