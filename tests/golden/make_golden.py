#!/usr/bin/env python3
"""Regenerate the golden fixtures in this directory from the reference repository.

Run where the reference tree is checked out ($BK_REFERENCE_ROOT, default /root/reference);
the GPU box never runs this. Every fixture is a small excerpt of a file the
reference itself ships:

* ``energy_exhaustive.json``  E(s) for every s at n = 1..12 and 1000 seeded rows at
  n = 16, 20 (C_1..C_{n-1}, E) from data_raw/classical/exhaustive/{n}.csv.
* ``min_energies.json``       data_raw/classical/exhaustive/min_energies.csv.
* ``traps.json``              trap rows of data_processed/probability_dynamics_n{N}_results.csv
                              and the orbit tables data_processed/exhaustive_minima_n{N}.json.
* ``series_n{N}.json``        P_<(t), <d_H(t)> series of selected (trap, g) pairs from
                              data_processed/probability_dynamics_n{N}.csv (cuStateVec
                              complex128 on H200, dt = 0.05, 1200 steps, every step);
                              N <= 20 keep every point, N >= 24 every 10th point.
* ``time_series_rows_n{N}.csv`` the header and selected rows, verbatim, of
                              data_processed/probability_dynamics_n{N}.csv (the connector's
                              export_time_series_csv output): the file's first row, rows across a
                              record boundary and rows with P_< > 0 — the byte-level pin of
                              bk_b200.export's time-series writer.
"""
import argparse
import csv
import json
import os
import random

SERIES = {  # N -> list of (trap_rank, g or None for all three g)
    16: [(8, None), (5, 0.35)],
    20: [(6, 0.35)],
    24: [(4, None)],
    26: [(3, None)],
    28: [(2, None)],
    30: [(2, None)],
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BK_REFERENCE_ROOT", "/root/reference"))
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    ex = os.path.join(a.ref, "data_raw/classical/exhaustive")
    dp = os.path.join(a.ref, "data_processed")

    energy = {"full": {}, "sampled": {}}
    for n in range(1, 13):
        rows = list(csv.reader(open(os.path.join(ex, f"{n}.csv"))))[1:]
        energy["full"][str(n)] = [int(r[-1]) for r in rows]
        assert [int(r[0]) for r in rows] == list(range(len(rows)))
    rng = random.Random(20240601)
    for n in (16, 20):
        want = set(rng.randrange(1 << n) for _ in range(1000))
        out = []
        with open(os.path.join(ex, f"{n}.csv")) as f:
            next(f)
            for line in f:
                s = line.split(",", 1)[0]
                if int(s) in want:
                    vals = [int(v) for v in line.strip().split(",")]
                    out.append(vals)
        energy["sampled"][str(n)] = out
    json.dump(energy, open(os.path.join(a.out, "energy_exhaustive.json"), "w"), separators=(",", ":"))

    # columns: n, E*(n), the lowest-index state reaching E*(n)
    mins = [dict(n=int(r["Mask"]), energy=int(r["Energy"]), first_state=int(r["N"]))
            for r in csv.DictReader(open(os.path.join(ex, "min_energies.csv")))]
    json.dump(mins, open(os.path.join(a.out, "min_energies.json"), "w"), indent=0)

    traps = {"results": {}, "orbits": {}}
    for n in (16, 20, 24, 26, 28, 30):
        rows = list(csv.DictReader(open(os.path.join(dp, f"probability_dynamics_n{n}_results.csv"))))
        keep = ("N", "g", "trap_rank", "trap_energy", "d_min", "window_avg_p_less", "window_avg_dh",
                "initial_rise_rate_avg", "initial_rise_rate_max", "peak_p_less", "peak_time",
                "p_blind", "quantum_time_sec", "trap_bits")
        traps["results"][str(n)] = [{k: r[k] for k in keep} for r in rows]
    for n in (20, 22, 24, 26, 28, 30):
        d = json.load(open(os.path.join(dp, f"exhaustive_minima_n{n}.json")))
        traps["orbits"][str(n)] = {"E_star": d["E_star"], "levels": [
            {"E0": l["E0"], "orbits": [{"canonical_id": o["canonical_id"], "bitstring": o["bitstring"],
                                        "d_min": o["d_min"]} for o in l["orbits"]]} for l in d["levels"]]}
    json.dump(traps, open(os.path.join(a.out, "traps.json"), "w"), indent=0)

    for n, picks in SERIES.items():
        res = {(int(r["trap_rank"]), float(r["g"])): r for r in traps["results"][str(n)]}
        series = {}
        with open(os.path.join(dp, f"probability_dynamics_n{n}.csv")) as f:
            for r in csv.DictReader(f):
                key = (int(r["trap_rank"]), float(r["g"]))
                if not any(key[0] == tr and (g is None or abs(key[1] - g) < 1e-12) for tr, g in picks):
                    continue
                s = series.setdefault(key, {"time": [], "p_less": [], "dh": []})
                s["time"].append(float(r["time"]))
                s["p_less"].append(float(r["p_less"]))
                s["dh"].append(float(r["dH"]))
        out = []
        for (rank, g), s in sorted(series.items()):
            step = 1 if n <= 20 else 10
            out.append({"N": n, "g": g, "trap_rank": rank, "trap_energy": int(res[(rank, g)]["trap_energy"]),
                        "trap_bits": res[(rank, g)]["trap_bits"], "dt": 0.05, "t_max": 60.0,
                        "every": step, "time": s["time"][::step], "p_less": s["p_less"][::step],
                        "dh": s["dh"][::step]})
        json.dump({"source": f"data_processed/probability_dynamics_n{n}.csv", "series": out},
                  open(os.path.join(a.out, f"series_n{n}.json"), "w"), separators=(",", ":"))
    for n in (16, 28):
        with open(os.path.join(dp, f"probability_dynamics_n{n}.csv"), newline="") as f:
            lines = f.read().split("\n")
        header, rows = lines[0], [x for x in lines[1:] if x]
        keep = list(range(12)) + list(range(1197, 1206))
        keep += [i for i, x in enumerate(rows) if float(x.split(",")[5]) > 0.0][:20] + [len(rows) - 2, len(rows) - 1]
        picked = [rows[i] for i in sorted(set(keep))]
        with open(os.path.join(a.out, f"time_series_rows_n{n}.csv"), "w", newline="") as f:
            f.write("\n".join([header] + picked) + "\n")
    print("golden fixtures written to", a.out)


if __name__ == "__main__":
    main()
