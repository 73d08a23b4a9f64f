"""Copies the input tables of PyPSA golden networks and the expected LOPF
results (objective, generator dispatch, line flows, storage trajectories,
optimal capacities and the objective constant) from the reference's
goldens (reference/goldens/{networks,results} in oluies/noaidi, generated by
PyPSA 1.2.4) into tests/golden/lopf/<network>/.

    python tests/golden/make_lopf_fixtures.py [path to the reference checkout]
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NETWORKS = ["ac-dc-dispatch", "ac-dc-co2", "lodf-mesh", "sclopf-triangle", "storage-cycle", "ac-dc-meshed", "storage-hvdc",
            "store-bank", "transformer-levels", "phase-shift"]
# input tables only: component lists, their input series and the snapshots
INPUTS = ["buses.csv", "carriers.csv", "generators.csv", "generators-p_max_pu.csv", "generators-p_min_pu.csv",
          "generators-marginal_cost.csv", "lines.csv", "links.csv", "loads.csv", "loads-p_set.csv", "snapshots.csv",
          "global_constraints.csv", "storage_units.csv", "storage_units-inflow.csv",
          "storage_units-state_of_charge_set.csv", "stores.csv", "transformers.csv"]


def main(root):
    goldens = os.path.join(root, "reference", "goldens")
    for name in NETWORKS:
        src = os.path.join(goldens, "networks", name)
        dst = os.path.join(HERE, "lopf", name)
        os.makedirs(dst, exist_ok=True)
        for f in INPUTS:
            if os.path.exists(os.path.join(src, f)):
                shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
        full = json.load(open(os.path.join(goldens, "results", f"{name}.json")))
        res = full["optimize"]
        keep = {k: res[k] for k in ("objective", "status", "condition", "generator_p", "line_p0", "link_p0",
                                    "storage_p_dispatch", "storage_p_store", "storage_state_of_charge",
                                    "storage_spill", "store_e", "store_p", "transformer_p0", "objective_constant", "total_system_cost", "nominal_opt")
                if k in res}
        if "sclopf" in full:  # the security-constrained solve, with the outages PyPSA used
            keep["sclopf"] = {k: full["sclopf"][k] for k in ("branch_outages", "objective", "status", "generator_p",
                                                             "line_p0")}
        with open(os.path.join(dst, "expected.json"), "w") as f:
            json.dump(keep, f, indent=1)
        print(name, "->", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
