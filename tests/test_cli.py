"""The lxmf-vanity command line (the reference's CLI surface, src/main.rs:325-499).

CPU tests cover argument handling and exit codes; GPU tests run real searches
and the self-test, and check the written identity file from scratch with the
oracle (address) and the file system (64 bytes, mode 0600, never overwritten)."""
import os
import re
import stat
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "lxmf-vanity_b200", "lxmf-vanity")


def run(args, cwd, timeout=300):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=timeout)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(CLI):
        pytest.fail(f"{CLI} is not built (python lxmf-vanity_b200/build.py)")


def test_usage_errors(tmp_path):
    for args in ([], ["--gpu"], ["--bogus", "b0"], ["--cpu", "b0"], ["--gpu", "b0", "c1"], ["--walk", "slow", "--gpu", "b0"]):
        r = run(args, tmp_path)
        assert r.returncode == 1 and "usage:" in r.stderr, args


def test_bad_prefix_is_refused(tmp_path):
    r = run(["--gpu", "BOOB"], tmp_path)
    assert r.returncode == 1
    assert "isn't 1 to 32 hex digits" in r.stderr and "not the letter O" in r.stderr
    r = run(["--gpu", "0" * 33], tmp_path)
    assert r.returncode == 1


def test_existing_identity_is_not_overwritten(tmp_path):
    p = tmp_path / "b00.identity"
    p.write_bytes(b"x" * 64)
    r = run(["--gpu", "B00"], tmp_path)
    assert r.returncode == 1 and "already exists; not overwriting it" in r.stderr
    assert p.read_bytes() == b"x" * 64


def test_no_gpu_reports_instead_of_crashing(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = run(["--gpu", "b0"], tmp_path)
    assert r.returncode == 2 and "unavailable" in r.stderr
    assert not (tmp_path / "b0.identity").exists()
    r = run(["--gpu-self-test"], tmp_path)
    assert r.returncode == 1 and "GPU unavailable" in r.stderr


def _check_identity(path, prefix, aspect="lxmf.delivery"):
    from oracle import oracle as O
    data = path.read_bytes()
    assert len(data) == 64
    assert stat.S_IMODE(os.stat(path).st_mode) == 0o600
    addr = O.address_of_identity(data, aspect)
    assert O.prefix_matches(O.prefix_parse(prefix), addr)
    return addr.hex()


def test_cpu_search_writes_a_valid_identity(tmp_path):
    r = run(["--threads", "2", "B0C"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Searching on 2 CPU threads; about 4096 tries on average." in r.stdout
    addr = _check_identity(tmp_path / "b0c.identity", "b0c")
    assert f"Found {addr}" in r.stdout
    assert re.search(r"About \d+ tries in [\d.]+ s \(\d+/s\)\. Saved to b0c\.identity", r.stdout)


def test_cpu_search_defaults_to_every_core(tmp_path):
    r = run(["b0"], tmp_path)
    assert r.returncode == 0, r.stderr
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    m = re.search(r"Searching on (\d+) CPU threads?;", r.stdout)
    assert m and int(m.group(1)) >= 1
    assert int(m.group(1)) <= max(cores, os.cpu_count() or 1)
    _check_identity(tmp_path / "b0.identity", "b0")


def test_seeded_cpu_search_finds_the_golden_hit(tmp_path):
    """One seeded thread walks seed 1's identity scalar: the golden first hit."""
    import json
    from oracle import oracle as O
    with open(os.path.join(ROOT, "tests", "golden", "config1.json")) as f:
        g = json.load(f)
    r = run(["--seed", str(g["seed"]), "--threads", "1", g["prefix"]], tmp_path)
    assert r.returncode == 0, r.stderr
    want = O.step_scalar(bytes.fromhex(g["scalar"]), g["hits"][0]) + bytes.fromhex(g["ed_seed"])
    assert (tmp_path / (g["prefix"] + ".identity")).read_bytes() == want
    assert f"About {g['hits'][0] + 1} tries" in r.stdout
    _check_identity(tmp_path / (g["prefix"] + ".identity"), g["prefix"])


def test_batch_file_errors(tmp_path):
    (tmp_path / "ok.txt").write_text("b0\nc1 nomadnetwork.node\n")
    for args in (["--batch-file", "ok.txt"], ["--gpu", "--cpu", "--batch-file", "ok.txt"],
                 ["--gpu", "--batch-file", "ok.txt", "b0"]):
        r = run(args, tmp_path)
        assert r.returncode == 1 and "usage:" in r.stderr, args
    cases = {
        "dup.txt": ("b0\nB0 lxmf.propagation\n", "listed twice"),
        "extra.txt": ("b0 lxmf.delivery extra\n", "expected '<hex prefix> [aspect]'"),
        "badhex.txt": ("# a comment\nbo\n", "isn't 1 to 32 hex digits"),
        "empty.txt": ("\n# nothing\n", "lists no searches"),
    }
    for name, (text, msg) in cases.items():
        (tmp_path / name).write_text(text)
        r = run(["--gpu", "--batch-file", name], tmp_path)
        assert r.returncode == 1 and msg in r.stderr, (name, r.stderr)
    r = run(["--gpu", "--batch-file", "missing.txt"], tmp_path)
    assert r.returncode == 1 and "could not read" in r.stderr
    (tmp_path / "c1.identity").write_bytes(b"y" * 64)
    r = run(["--gpu", "--batch-file", "ok.txt"], tmp_path)
    assert r.returncode == 1 and "c1.identity already exists" in r.stderr
    assert (tmp_path / "c1.identity").read_bytes() == b"y" * 64


BATCH_LINES = ["b0b", "c0ffe nomadnetwork.node", "d1 lxmf.propagation", "A2C4"]


@pytest.mark.gpu
def test_batch_file_saves_every_identity(tmp_path):
    (tmp_path / "list.txt").write_text("\n".join(BATCH_LINES) + "\n")
    r = run(["--gpu", "--batch-file", "list.txt"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "4 searches on the GPU pool" in r.stdout and "All 4 found" in r.stdout
    for line in BATCH_LINES:
        prefix, *aspect = line.lower().split()
        addr = _check_identity(tmp_path / f"{prefix}.identity", prefix, *(aspect or ["lxmf.delivery"]))
        assert f"Found {addr}" in r.stdout


@pytest.mark.gpu
def test_batch_file_results_are_the_same_alone_and_in_the_mix(tmp_path):
    """Seeded: search i of the file uses seed N + i, and every lane of the pool
    advances in step, so each search's identity is the one it finds alone."""
    mix = tmp_path / "mix"
    mix.mkdir()
    (mix / "list.txt").write_text("\n".join(BATCH_LINES) + "\n")
    r = run(["--gpu", "--seed", "77", "--batch-file", "list.txt"], mix)
    assert r.returncode == 0, r.stderr
    for i, line in enumerate(BATCH_LINES):
        alone = tmp_path / f"alone{i}"
        alone.mkdir()
        (alone / "one.txt").write_text(line + "\n")
        r = run(["--gpu", "--seed", str(77 + i), "--batch-file", "one.txt"], alone)
        assert r.returncode == 0, r.stderr
        prefix = line.split()[0].lower()
        assert (alone / f"{prefix}.identity").read_bytes() == (mix / f"{prefix}.identity").read_bytes(), line


@pytest.mark.gpu
def test_two_replicas_on_one_device(tmp_path):
    """--devices 0,0: two independent handles (seeds N and N + 1), first hit wins."""
    r = run(["--gpu", "--devices", "0,0", "--seed", "9", "--lanes", "8192", "b00b"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Searching on 2 GPUs" in r.stdout
    _check_identity(tmp_path / "b00b.identity", "b00b")


@pytest.mark.gpu
def test_gpu_and_cpu_together(tmp_path):
    r = run(["--gpu", "--cpu", "--threads", "2", "B00B"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Searching on 1 GPU and 2 CPU threads" in r.stdout
    addr = _check_identity(tmp_path / "b00b.identity", "b00b")
    assert f"Found {addr}" in r.stdout


@pytest.mark.gpu
def test_self_test_passes(tmp_path):
    # 256 lanes x one batch of keys each: the default 1024, and the reference's 64 (mod.rs:178-207).
    for args, keys in (([], 256 * 1024), (["--batch", "64"], 256 * 64)):
        r = run(["--gpu-self-test"] + args, tmp_path)
        assert r.returncode == 0, r.stderr
        m = re.search(r"Self-test passed: (\d+) public keys match X25519, (\d+) hits", r.stdout)
        assert m and int(m.group(1)) == keys and int(m.group(2)) >= 100


@pytest.mark.gpu
@pytest.mark.parametrize("walk", ["group", "xadd"])
def test_search_writes_a_valid_identity(tmp_path, walk):
    r = run(["--gpu", "--walk", walk, "B00B"], tmp_path)
    assert r.returncode == 0, r.stderr
    addr = _check_identity(tmp_path / "b00b.identity", "b00b")
    assert f"Found {addr}" in r.stdout
    assert re.search(r"About \d+ tries in [\d.]+ s \(\d+/s\)\. Saved to b00b\.identity", r.stdout)
    r = run(["--gpu", "b00b"], tmp_path)
    assert r.returncode == 1 and "already exists" in r.stderr


@pytest.mark.gpu
def test_seeded_search_is_reproducible_and_honours_the_aspect(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    for d in (a, b):
        r = run(["--gpu", "--seed", "12345", "--aspect", "nomadnetwork.node", "--lanes", "8192", "abc"], d)
        assert r.returncode == 0, r.stderr
    assert (a / "abc.identity").read_bytes() == (b / "abc.identity").read_bytes()
    _check_identity(a / "abc.identity", "abc", "nomadnetwork.node")
