"""The OBJ reader reads a large file in pieces on several threads (host, CPU only).

A first pass counts each piece's lines, vertices, texture coordinates and
triangles; a second reads every piece with the counts of the lines before it.
tests/cpp/obj_pieces.cpp compiles the reader's own source and reads each file in
1, 2, 3, 5, 8 and 13 pieces, comparing the meshes (a hash of every coordinate
and index) or the error messages. The files are seeded mutations of OBJ texts
that use every statement the reader knows (v, vt, f with and without texture
indices, negative indices, comments, CRLF line ends, a last line without a line
end), so pieces begin and end at every kind of line and errors fall in every
piece. Budgets below the files' sizes make the vertex, texture-coordinate and
triangle limits fail part-way through. The one-piece reader is the reference's
(tests/test_reader_parity.py compares it with readScene).
"""

import random
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "albedo_b200" / "csrc"
BIG = 1 << 24


def generated_obj(rng: random.Random, vertices: int = 400) -> str:
    lines = ["# generated mesh", ""]
    for i in range(vertices):
        lines.append(f"v {rng.uniform(-5, 5):.6f} {rng.uniform(-5, 5):.6f} {rng.uniform(-5, 5):.6f}")
        if i % 3 == 0:
            lines.append(f"vt {rng.random():.4f} {rng.random():.4f}")
        if i >= 3 and i % 2 == 0:
            a, b, c = rng.sample(range(1, i + 1), 3)
            textures = (i // 3) + 1
            form = rng.randrange(4)
            if form == 0:
                lines.append(f"f {a} {b} {c}")
            elif form == 1:
                t = [rng.randrange(1, textures + 1) for _ in range(3)]
                lines.append(f"f {a}/{t[0]} {b}/{t[1]} {c}/{t[2]}  # textured")
            elif form == 2:
                lines.append(f"f -1 -2 -3 {-rng.randrange(4, i + 1)}")
            else:
                lines.append(f"f {a}//{a} {b}//{b} {c}//{c}")
    text = "\r\n".join(lines[: len(lines) // 2]) + "\r\n" + "\n".join(lines[len(lines) // 2:])
    return text  # the last line has no line end


KNOT = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0.5 0.5 1\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n" \
       "f 1/1 2/2 5/3\nf 2/2 3/3 5/3\nf 3/3 4/4 5/3\nf 4/4 1/1 5/3\nf 1 2 3 4\n"

BAD = ["nan", "-1", "0", "1e400", "abc", "3.5", "-0", "inf", "99999", "1/0", "//", "-99"]


def mutate(text: str, rng: random.Random) -> str:
    lines = text.split("\n")
    for _ in range(rng.randrange(1, 4)):
        i = rng.randrange(len(lines))
        words = lines[i].split(" ")
        kind = rng.randrange(6)
        if kind == 0:
            del lines[i]
        elif kind == 1:
            lines.insert(i, lines[i])
        elif kind == 2 and len(words) > 1:
            del words[rng.randrange(1, len(words))]
            lines[i] = " ".join(words)
        elif kind == 3 and len(words) > 1:
            words[rng.randrange(1, len(words))] = rng.choice(BAD)
            lines[i] = " ".join(words)
        elif kind == 4:
            lines[i] = lines[i] + " " + rng.choice(["junk", "1", "#", "nan"])
        else:
            j = rng.randrange(len(lines))
            lines[i], lines[j] = lines[j], lines[i]
        if not lines:
            lines = [""]
    return "\n".join(lines)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("obj") / "obj_pieces"
    subprocess.run(["g++", "-std=c++20", "-O1", "-ffp-contract=off", f"-I{CSRC}", str(HERE / "cpp" / "obj_pieces.cpp"),
                    str(CSRC / "host" / "bvh_build.cpp"), str(CSRC / "host" / "host_math.cpp"),
                    str(CSRC / "host" / "host_scene.cpp"), "-pthread", "-o", str(exe)], check=True)
    return exe


def run(harness, cases):
    args = []
    for path, budget in cases:
        args += [str(path), *(str(b) for b in budget)]
    out = subprocess.run([str(harness), *args], check=True, capture_output=True, text=True).stdout.splitlines()
    assert len(out) == len(cases)
    return [line.split("\t", 1) for line in out]


@pytest.mark.parametrize("base", ["knot", "generated"])
def test_pieces_read_like_one_thread(tmp_path, harness, base):
    rng = random.Random({"knot": 3, "generated": 4}[base])
    cases = []
    for k in range(200):
        text = KNOT if base == "knot" else generated_obj(rng)
        if k > 0:
            text = mutate(text, rng)
        path = tmp_path / f"case{k}.obj"
        path.write_bytes(text.encode())
        budget = (BIG, BIG, BIG)
        if k % 5 == 4:
            budget = (rng.randrange(3, 300), BIG, BIG)
        elif k % 5 == 3:
            budget = (BIG, rng.randrange(0, 100), rng.randrange(1, 200))
        cases.append((path, budget))
    results = run(harness, cases)
    assert all(same == "same" for same, _ in results), [r for r in results if r[0] != "same"][:3]
    outcomes = [outcome.split(" ")[0] for _, outcome in results]
    assert outcomes.count("ok") > 20 and outcomes.count("error") > 20
    messages = " ".join(outcome for _, outcome in results)
    if base == "generated":
        for problem in ("more than", "not yet defined", "not a finite number", "not a valid index"):
            assert problem in messages, problem


def test_a_file_without_lines_and_a_file_of_one_line(tmp_path, harness):
    cases = []
    for k, text in enumerate(["", "\n", "v 1 2 3", "v 1 2 3\n\n\n", "\n\n\nf 1 2 3\n"]):
        path = tmp_path / f"edge{k}.obj"
        path.write_bytes(text.encode())
        cases.append((path, (BIG, BIG, BIG)))
    results = run(harness, cases)
    assert all(same == "same" for same, _ in results), results
    assert results[4][1] == "error OBJ line 4: a face refers to a vertex not yet defined"
