"""Restart files in the reference's MPCNSRST version 1 format
(src/6_io/IOModule_Bin.cpp:168-420), host side: the library's reader
(mhd_restart_read) against a file the reference's own writer produced after
a few steps (its state is also dumped, so every value is checked, ghosts
included), and the library's writer (mhd_restart_write) against the same
file byte for byte.  Malformed files are rejected with MHD_ERR_ARG."""
import struct

import numpy as np
import pytest

N = 6
NGHOST = 4
STEPS = 3


@pytest.fixture(scope="module")
def ref_restart(ref_oracle, tmp_path_factory):
    d = tmp_path_factory.mktemp("restart")
    path = str(d / "ref.bin")
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=N, steps=STEPS, dump_at=str(STEPS), write_restart=path,
               dump_fields=" ".join(ref_oracle.STATE_FIELDS))
    dump = ref_oracle.run_job(job, workdir=str(d / "job"))
    return path, dump


def test_reader_matches_reference_state(ref_restart):
    from mpcns_mercury_b200 import capi

    path, dump = ref_restart
    step, time, fields = capi.restart_read(path, [(N, N, N)], NGHOST)
    assert step == STEPS
    assert time == dump[(f"step{STEPS}:dt_time", -1)].data.ravel()[1]
    assert sorted(fields) == sorted(capi.RESTART_FIELDS)
    for name in capi.RESTART_FIELDS:
        ref = dump[(f"step{STEPS}:{name}", 0)]
        assert tuple(ref.lo) == (-NGHOST,) * 3
        got = fields[name][0]
        assert got.shape == ref.data.shape, name
        assert np.array_equal(got, ref.data), name


def test_writer_reproduces_reference_file(ref_restart, tmp_path):
    from mpcns_mercury_b200 import capi

    path, _ = ref_restart
    step, time, fields = capi.restart_read(path, [(N, N, N)], NGHOST)
    out = str(tmp_path / "ours.bin")
    capi.restart_write(out, step, time, [(N, N, N)], NGHOST, fields)
    with open(path, "rb") as a, open(out, "rb") as b:
        assert a.read() == b.read()


def _fields_of(path):
    """(header bytes, [(name, field bytes)]) of a one-block restart file."""
    raw = open(path, "rb").read()
    head = raw[:8 + 4 + 4 + 8 + 4 + 4]
    nfield = struct.unpack_from("<i", raw, 28)[0]
    pos, out = len(head), []
    for _ in range(nfield):
        start = pos
        ln = struct.unpack_from("<i", raw, pos)[0]
        name = raw[pos + 4:pos + 4 + ln].decode()
        pos += 4 + ln
        _, ncomp, _ = struct.unpack_from("<iii", raw, pos)
        pos += 12
        lo = struct.unpack_from("<3i", raw, pos)
        hi = struct.unpack_from("<3i", raw, pos + 12)
        pos += 28
        pos += 8 * int(np.prod(np.subtract(hi, lo))) * ncomp
        out.append((name, raw[start:pos]))
    return head, out


def _assemble(head, parts):
    return head[:28] + struct.pack("<i", len(parts)) + b"".join(p for _, p in parts)


def test_reader_skips_unknown_and_reports_missing(ref_restart, tmp_path):
    """Fields the library does not restore are skipped; fields the file lacks
    are reported absent (the reference keeps their current values)."""
    from mpcns_mercury_b200 import capi

    path, dump = ref_restart
    head, parts = _fields_of(path)
    extra = bytearray(parts[2][1])             # B_xi's record renamed: an unknown field
    extra[4:8] = b"X_xi"
    mixed = [parts[0], ("X_xi", bytes(extra)), parts[1], parts[2], parts[3]]  # no B_zeta
    p = str(tmp_path / "mixed.bin")
    open(p, "wb").write(_assemble(head, mixed))
    _, _, fields = capi.restart_read(p, [(N, N, N)], NGHOST)
    assert sorted(fields) == sorted(["U_H", "U_Na", "B_xi", "B_eta"])
    assert np.array_equal(fields["U_Na"][0], dump[(f"step{STEPS}:U_Na", 0)].data)


@pytest.mark.parametrize("case", ["magic", "version", "blocks", "nghost", "range", "truncated", "location"])
def test_reader_rejects_malformed(ref_restart, tmp_path, case):
    from mpcns_mercury_b200 import capi

    path, _ = ref_restart
    raw = bytearray(open(path, "rb").read())
    cells, nghost = [(N, N, N)], NGHOST
    if case == "magic":
        raw[0:8] = b"MPCNSRSX"
    elif case == "version":
        raw[8:12] = struct.pack("<i", 2)
    elif case == "blocks":
        cells = [(N, N, N), (N, N, N)]
    elif case == "nghost":
        nghost = NGHOST - 1
    elif case == "range":
        cells = [(N, N, N + 1)]
    elif case == "truncated":
        raw = raw[:len(raw) - 100]
    elif case == "location":
        ln = struct.unpack_from("<i", raw, 32)[0]
        raw[36 + ln:40 + ln] = struct.pack("<i", 1)  # U_H claimed face-centred
    p = str(tmp_path / f"{case}.bin")
    open(p, "wb").write(bytes(raw))
    with pytest.raises(capi.MhdError) as e:
        capi.restart_read(p, cells, nghost)
    assert "ERR_ARG" in str(e.value) and "mhd_restart_read:" in str(e.value)


@pytest.fixture(scope="module")
def ref_lattice_restart(ref_oracle, tmp_path_factory):
    d = tmp_path_factory.mktemp("restart_lattice")
    path = str(d / "ref.bin")
    job = dict(ref_oracle.CUBE_JOB)
    job.update(case="lattice", n=4, nb="2 2 2", steps=2, dump_at="2", write_restart=path,
               dump_fields=" ".join(ref_oracle.STATE_FIELDS))
    dump = ref_oracle.run_job(job, workdir=str(d / "job"))
    return path, dump


def test_multi_block_restart_matches_reference(ref_lattice_restart, tmp_path):
    """Eight blocks of a periodic box (the reference's lattice case after 2
    steps): every block's values read back, ghosts included, and the file
    written again byte for byte."""
    from mpcns_mercury_b200 import capi

    path, dump = ref_lattice_restart
    cells = [(4, 4, 4)] * 8
    step, time, fields = capi.restart_read(path, cells, NGHOST)
    assert step == 2
    for name in capi.RESTART_FIELDS:
        for b in range(8):
            ref = dump[(f"step2:{name}", b)]
            assert np.array_equal(fields[name][b], ref.data), (name, b)
    out = str(tmp_path / "ours.bin")
    capi.restart_write(out, step, time, cells, NGHOST, fields)
    with open(path, "rb") as a, open(out, "rb") as c:
        assert a.read() == c.read()


def test_rundata_file_matches_reference(ref_oracle, tmp_path):
    """The run-data file beside a checkpoint (RunData::WriteBinary) from the
    run's step, time and last dt, byte for byte against the reference's, and
    read back."""
    from mpcns_mercury_b200 import capi

    ref = str(tmp_path / "ref.bin")
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=N, steps=STEPS, dump_at=str(STEPS), write_rundata=ref, dump_fields="U_H")
    dump = ref_oracle.run_job(job, workdir=str(tmp_path / "job"))
    dt, time = dump[(f"step{STEPS}:dt_time", -1)].data.ravel()
    # the monitors are the run's wall-clock performance figures: taken from
    # the reference's file (the format is what is checked)
    raw = open(ref, "rb").read()
    p = 8 + 4 + 4 + 8 + 8
    nref = struct.unpack_from("<i", raw, p)[0]
    p += 4 + 8 * nref + 8
    mons = []
    for fmt, size in (("<d", 8), ("<i", 4)):
        n = struct.unpack_from("<i", raw, p)[0]
        p += 4
        m = {}
        for _ in range(n):
            ln = struct.unpack_from("<i", raw, p)[0]
            key = raw[p + 4:p + 4 + ln].decode()
            m[key] = struct.unpack_from(fmt, raw, p + 4 + ln)[0]
            p += 4 + ln + size
        mons.append(m)
    assert sorted(mons[0]) == ["Perf/CPUInterval_s", "Perf/s_per_MCells_step"] and list(mons[1]) == ["Perf/Cells"]
    assert mons[1]["Perf/Cells"] == N ** 3
    ours = str(tmp_path / "ours.bin")
    # keys given out of order: the writer orders them as the reference's map does
    capi.rundata_write(ours, STEPS, time, dt, monitors_d=dict(reversed(list(mons[0].items()))),
                       monitors_i={"Perf/Cells": N ** 3})
    with open(ref, "rb") as a, open(ours, "rb") as b:
        assert a.read() == b.read()
    assert capi.rundata_read(ref) == (STEPS, time, dt)
