"""The resident environment server (phop_resident_serve, parahpop_gpu --serve):
command-line runs forwarded over a Unix-domain socket to a process that
keeps their environments on the device.  The protocol, the refusals and the
driver's own error text through the server are checked on the CPU (the
driver fails there at its device check, after the request has crossed the
socket); results and reuse of a kept environment on the GPU."""
import json
import os
import subprocess
import time

import numpy as np
import pytest

from parahpop_b200 import api


class ResidentServer:
    def __init__(self, sock):
        self.sock = str(sock)
        self.proc = subprocess.Popen([str(api.CLI_PATH), "--serve", self.sock], stdout=subprocess.PIPE,
                                     stderr=subprocess.PIPE, text=True)
        for _ in range(400):
            if os.path.exists(self.sock) or self.proc.poll() is not None:
                break
            time.sleep(0.05)
        assert os.path.exists(self.sock), self.proc.stderr.read() if self.proc.poll() is not None else "no socket"

    def env(self, **extra):
        return dict(os.environ, PARAHPOP_B200_SERVER=self.sock, **extra)

    def stop(self):
        r = subprocess.run([str(api.CLI_PATH), "--stop", self.sock], capture_output=True, text=True, timeout=60)
        rc = self.proc.wait(timeout=60)
        return r.returncode, rc

    def kill(self):
        if self.proc.poll() is None:
            self.proc.kill()
            self.proc.wait(timeout=30)


@pytest.fixture
def server(tmp_path):
    s = ResidentServer(tmp_path / "phop.sock")
    yield s
    s.kill()


def test_protocol_and_refusals(golden, server, tmp_path):
    case = golden("full_600s")
    # a second server on the same socket is refused while the first answers
    r = subprocess.run([str(api.CLI_PATH), "--serve", server.sock], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "a server already answers at" in r.stderr
    # the driver's argument checks run in the server and come back verbatim
    r = api.run_cli(case.config_path, case.targets_path, tmp_path / "out", env=server.env())
    if r.returncode != 0:  # no CUDA device here: the driver's own device message, from the server
        assert r.stderr.startswith("ParaHPOP: No usable CUDA device")
    existing = tmp_path / "existing"
    existing.mkdir()
    (existing / "summary.json").write_text("{}")
    r = api.run_cli(case.config_path, case.targets_path, existing, env=server.env())
    assert r.returncode == 1
    assert r.stderr.startswith("ParaHPOP: Output exists; use a new directory:")
    assert server.stop() == (0, 0)
    assert not os.path.exists(server.sock)


def test_client_without_server(golden, tmp_path):
    case = golden("full_600s")
    sock = tmp_path / "nobody.sock"
    r = api.run_cli(case.config_path, case.targets_path, tmp_path / "out", env=dict(os.environ,
                                                                                    PARAHPOP_B200_SERVER=str(sock)))
    assert r.returncode == 1
    assert r.stderr.startswith(f"ParaHPOP: no resident environment server answers at {sock}")
    assert subprocess.run([str(api.CLI_PATH), "--stop", str(sock)]).returncode == 1


def _states(out):
    return np.loadtxt(out / "final_states.csv", delimiter=",", skiprows=1)


def _summary(out):
    return json.loads((out / "summary.json").read_text())


@pytest.mark.gpu
def test_kept_environment_runs_match_in_process_runs(golden, server, tmp_path):
    case = golden("full_600s")
    pinned = {"PARAHPOP_B200_LANES": "2"}
    ref = api.run_cli(case.config_path, case.targets_path, tmp_path / "inproc", env=dict(os.environ, **pinned))
    assert ref.returncode == 0, ref.stderr
    first = api.run_cli(case.config_path, case.targets_path, tmp_path / "first", env=server.env(**pinned))
    second = api.run_cli(case.config_path, case.targets_path, tmp_path / "second", env=server.env(**pinned))
    assert first.returncode == 0 and second.returncode == 0, first.stderr + second.stderr
    # the summary is echoed to the client's standard output, as the driver does
    assert json.loads(second.stdout) == _summary(tmp_path / "second")
    np.testing.assert_array_equal(_states(tmp_path / "first"), _states(tmp_path / "inproc"))
    np.testing.assert_array_equal(_states(tmp_path / "second"), _states(tmp_path / "inproc"))
    assert (tmp_path / "second" / "configuration_resolved.json").read_text() == \
        (tmp_path / "inproc" / "configuration_resolved.json").read_text()
    # the second run found the environment on the device
    assert _summary(tmp_path / "second")["environment_seconds"] < _summary(tmp_path / "first")["environment_seconds"]
    # a data file that changed is loaded again (the results stay the same)
    st = os.stat(case.dir / "gravity.tab")
    os.utime(case.dir / "gravity.tab", ns=(st.st_atime_ns, st.st_mtime_ns + 10 ** 9))
    third = api.run_cli(case.config_path, case.targets_path, tmp_path / "third", env=server.env(**pinned))
    assert third.returncode == 0, third.stderr
    np.testing.assert_array_equal(_states(tmp_path / "third"), _states(tmp_path / "inproc"))
    # the golden's reference states hold through the server
    assert np.abs(_states(tmp_path / "second")[:, 2:5] - np.array(case.data["reference"]["states"])[:, :3]).max() < 1e-6
    # precision settings of the client reach the server
    split = api.run_cli(case.config_path, case.targets_path, tmp_path / "split",
                        env=server.env(PARAHPOP_B200_SPLIT="1", **pinned))
    assert split.returncode == 0, split.stderr
    assert np.abs(_states(tmp_path / "split")[:, 2:5] - _states(tmp_path / "inproc")[:, 2:5]).max() < 1e-5
    assert server.stop() == (0, 0)


def _exchange(sock_path, payload: bytes) -> dict:
    import socket
    import struct
    s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    s.settimeout(30)
    s.connect(sock_path)
    s.sendall(struct.pack("<I", len(payload)) + payload)
    n = struct.unpack("<I", s.recv(4, socket.MSG_WAITALL))[0]
    data = b""
    while len(data) < n:
        data += s.recv(n - len(data))
    s.close()
    return json.loads(data)


def test_malformed_requests_are_answered(server):
    """A request that is not the protocol's JSON gets a failure answer and
    the server keeps serving; a run request with the wrong number of paths
    gets the driver's own message."""
    bad = _exchange(server.sock, b"this is not json")
    assert bad["status"] == 1 and bad["stderr"].startswith("ParaHPOP: ")
    missing = _exchange(server.sock, json.dumps({"args": ["only-one"], "split": -1, "lanes": 0}).encode())
    assert missing["status"] == 1
    assert missing["stderr"].startswith("ParaHPOP: Expected CONFIG.json TARGETS.json OUTPUT_DIRECTORY")
    assert server.stop() == (0, 0)
