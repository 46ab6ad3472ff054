"""native.build() under concurrent processes: a builder waits for the lock
another holds, then re-checks and does not rebuild a library that became
current meanwhile; builders without a lock work in private directories.  The
compiler itself is stubbed out: no nvcc runs here."""
import fcntl
import os
import subprocess
import sys
import threading
import time

from hashpoint import native

CHILD = r"""
import sys, time
sys.path.insert(0, sys.argv[1])
from hashpoint import native
calls = []
def needs_build():
    calls.append(time.time())
    return len(calls) == 1          # stale before the lock, current after it
def build_locked(verbose, extra_flags):
    raise SystemExit("rebuilt a current library")
native.needs_build = needs_build
native._build_private = build_locked
print(native.build() == native.LIB_PATH, len(calls), "%.6f" % calls[-1])
"""


def test_second_builder_waits_and_skips_a_current_library():
    os.makedirs(native.LIB_DIR, exist_ok=True)
    pkg = os.path.dirname(os.path.dirname(os.path.abspath(native.__file__)))
    with open(os.path.join(native.LIB_DIR, ".build.lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        child = subprocess.Popen([sys.executable, "-c", CHILD, pkg], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                 text=True)
        time.sleep(1.0)
        assert child.poll() is None  # blocked on the lock
        released = time.time()
        fcntl.flock(lock, fcntl.LOCK_UN)
    out, err = child.communicate(timeout=60)
    assert child.returncode == 0, err
    ok, n_checks, t_second = out.split()
    assert ok == "True" and n_checks == "2"
    assert float(t_second) >= released - 0.05  # the re-check came after the lock was released


def test_builds_without_a_lock_where_the_filesystem_has_none(monkeypatch):
    calls = []

    def no_locks(*a):
        raise OSError("locks not supported")

    monkeypatch.setattr(native.fcntl, "flock", no_locks)
    monkeypatch.setattr(native, "needs_build", lambda: True)
    monkeypatch.setattr(native, "_build_private", lambda verbose, extra: calls.append(1) or native.LIB_PATH)
    assert native.build() == native.LIB_PATH and calls == [1]


def test_unlocked_builders_at_once_keep_their_files_apart(monkeypatch, tmp_path):
    """Two builders with no lock between them: each compiles and links in its own directory, so
    neither links or deletes the other's objects, and the library ends up whole."""
    lib = tmp_path / native.LIB_NAME
    monkeypatch.setattr(native, "LIB_DIR", str(tmp_path))
    monkeypatch.setattr(native, "LIB_PATH", str(lib))
    seen = []

    class Done:
        returncode, stdout = 0, ""

    def fake_run(cmd, **kw):
        out = cmd[cmd.index("-o") + 1]
        seen.append(os.path.dirname(out))
        if "-shared" in cmd:  # the link reads every object of its own build
            for o in cmd[cmd.index("-o") + 2:]:
                if o.endswith(".o"):
                    assert open(o).read() == "obj:" + os.path.dirname(out)
        time.sleep(0.05)
        with open(out, "w") as f:
            f.write("obj:" + os.path.dirname(out) if out.endswith(".o") else "library")
        return Done()

    monkeypatch.setattr(native.subprocess, "run", fake_run)
    errors = []

    def builder():
        try:
            assert native._build_private(False, ()) == str(lib)
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append(e)

    threads = [threading.Thread(target=builder) for _ in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(60)
    assert not errors, errors
    assert lib.read_text() == "library"
    assert len(set(seen)) == 2  # two private directories
    assert not [p for p in os.listdir(tmp_path) if p.startswith(".build-")]  # both cleaned up
