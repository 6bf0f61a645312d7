"""CEB query 1a: the plain-Python restatement (tests/ceb_restate.py) against
the reference itself -- its CEB load / build / query compiled unchanged into
oracle/_ref/ref_ceb_driver -- on seeded IMDB-shaped Parquet files
(bespokeolap_artifacts_b200.ceb_data), with and without nulls.  CPU only."""
import csv
import subprocess
from pathlib import Path

import pytest

from bespokeolap_artifacts_b200.ceb_data import write_ceb
from ceb_restate import q1a

ROOT = Path(__file__).resolve().parent.parent
REF_CEB = ROOT / "oracle" / "_ref" / "ref_ceb_driver"

# (ID1, ID2, INFO1, INFO2, KIND, ROLE, GENDER, YEAR1, YEAR2)
Q1A_CASES = [
    (["1", "2", "3", "5"], ["7", "8", "9"], ["V000", "V001", "V005"], ["V002", "V003"],
     ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B", "ROLE_D"], ["GENDER_F", "GENDER_M"], "2015", "1950"),
    (["1"], ["2"], ["V000"], ["V000"], ["KIND_A"], ["ROLE_A"], ["GENDER_F"], "2020", "1880"),
    (["1", "1"], ["1"], ["V000", "V001"], ["V001", "V000"], ["KIND_A", "KIND_G"], ["ROLE_L"], ["GENDER_M"],
     "1990", "1990"),
    (["114", "116", "NULL", "2x"], ["2", "-1"], ["V000", "NOSUCH"], ["V004", "<<NULL>>"], ["KIND_D", "NOSUCH"],
     ["ROLE_C", "ROLE_E"], ["GENDER_F"], "2020", "1880"),
    (["3"], ["4"], ["V010"], ["V011"], ["NOSUCH"], ["ROLE_A"], ["GENDER_F"], "2020", "1880"),
    (["1", "2"], ["3", "4"], ["V000", "V001"], ["V002", "V003"], ["KIND_A", "KIND_B"], ["ROLE_A"], ["GENDER_M"],
     "1900", "2000"),
]


def lit(vals):
    return "(" + ", ".join("'" + v.replace("'", "''") + "'" for v in vals) + ")"


def request(case) -> str:
    id1, id2, i1, i2, k, r, g, y1, y2 = case
    return f'1a {lit(id1)} {lit(id2)} {lit(i1)} {lit(i2)} {lit(k)} {lit(r)} {lit(g)} "{y1}" "{y2}"'


def reference(data: Path, workdir: Path, requests: list[str]) -> list[list[list[str]]]:
    workdir.mkdir(parents=True, exist_ok=True)
    p = subprocess.run([str(REF_CEB), str(data) + "/"], input="\n".join(requests) + "\n\n", text=True,
                       capture_output=True, cwd=workdir, timeout=300)
    assert p.returncode == 0, p.stderr
    return [list(csv.reader(open(workdir / f"result{i + 1}.csv"))) for i in range(len(requests))]


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2)])
def test_q1a_restatement_matches_reference(tmp_path, nulls, seed):
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls)
    got = reference(data, tmp_path / "ref", [request(c) for c in Q1A_CASES])
    nonzero = 0
    for case, g in zip(Q1A_CASES, got):
        assert g[0] == ["count_star()"]
        want = q1a(data, *case)
        assert int(g[1][0]) == want, case
        nonzero += want > 0
    assert nonzero >= 3


# (ID, INFO, NAME, KIND, ROLE)
Q10A_CASES = [
    (["1", "2", "3", "5"], ["V000", "V001", "V005"], "%00%", ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B"]),
    (["1"], ["V000", "V002"], "name_000%", ["KIND_A", "KIND_D"], ["ROLE_A", "ROLE_C", "ROLE_D"]),
    (["2", "3"], ["V001"], "%7", ["KIND_B"], ["ROLE_B"]),
    (["1", "4"], ["V000", "V003"], "%", ["KIND_A"], ["ROLE_A"]),
    (["1", "2"], ["V000"], "n_me_0_0%1", ["KIND_A", "KIND_B"], ["ROLE_A", "ROLE_E"]),
    (["1"], ["V000"], "'NAME_0000014'", ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B", "ROLE_C"]),
    (["x"], ["V000"], "%", ["KIND_A"], ["ROLE_A"]),
    (["1"], ["NOSUCH"], "%", ["KIND_A"], ["ROLE_A"]),
]


def request10a(case) -> str:
    ids, infos, name, kinds, roles = case
    return f'10a {lit(ids)} {lit(infos)} "{name}" {lit(kinds)} {lit(roles)}'


def q10a_csv_rows(g):
    """The reference's 10a CSV rows as (name, info, min, max), sorted (its
    row order is its aggregation order)."""
    return sorted((r[0], r[1], int(r[2]) if r[2] else None, int(r[3]) if r[3] else None) for r in g[1:])


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2)])
def test_q10a_restatement_matches_reference(tmp_path, nulls, seed):
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    from bespokeolap_artifacts_b200.ceb import string_pool
    from ceb_restate import q10a

    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls)
    pool = string_pool(data)
    got = reference(data, tmp_path / "ref", [request10a(c) for c in Q10A_CASES])
    nonempty = 0
    for case, g in zip(Q10A_CASES, got):
        assert g[0] == ["name", "info", "min(t.production_year)", "max(t.production_year)"]
        want = q10a(data, *case, pool)
        assert q10a_csv_rows(g) == want, case
        nonempty += len(want) > 0
    assert nonempty >= 4


# (TITLE, NAME_PCODE_NF, NAME, KIND, ROLE)
Q3B_CASES = [
    ("%1%", "a%", "%00%", ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B", "ROLE_C"]),
    ("title_1%", "%", "comp_%", ["KIND_A"], ["ROLE_A", "ROLE_D"]),
    ("%", "_1%", "%5", ["KIND_B", "KIND_C", "KIND_D"], ["ROLE_B"]),
    ("%2", "b%", "comp_0000%", ["KIND_A", "KIND_B"], ["ROLE_A", "ROLE_B", "ROLE_C", "ROLE_D"]),
    ("%", "%", "nosuch%", ["KIND_A"], ["ROLE_A"]),
]


def request3b(case) -> str:
    title, pcode, company, kinds, roles = case
    return f'3b "{title}" "{pcode}" "{company}" {lit(kinds)} {lit(roles)}'


def q3b_csv_rows(g):
    return [(r[0], r[1], r[2], int(r[3])) for r in g[1:]]


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2)])
def test_q3b_restatement_matches_reference(tmp_path, nulls, seed):
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    from ceb_restate import q3b

    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls, n_company=500, n_movie_companies=12_000, n_keyword=800, n_movie_keyword=15_000)
    got = reference(data, tmp_path / "ref", [request3b(c) for c in Q3B_CASES])
    nonempty = 0
    for case, g in zip(Q3B_CASES, got):
        assert g[0] == ["title", "name", "name_1", "count_star()"]
        want = q3b(data, *case)
        assert q3b_csv_rows(g) == want, case
        nonempty += len(want) > 0
    assert nonempty >= 3
