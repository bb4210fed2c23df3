"""Write the benchmark's default workload in the reference's own input format.

The obstacle-flow workload of bench.py is two cases — 256 x 256 cells, ngrid 5,
red-black Gauss-Seidel, a seeded staggered lattice of blocks on a 16 x 16 base grid
(porosity 0.75), Re 10 and Re 100 — each kept here as the InputData + pattern.txt
pair the reference program reads from its working directory (readInput,
Version-6-26-04.c:280-401; read_obstacle_data :2367-2400):

    workloads/obstacle256_re10/{InputData,pattern.txt}
    workloads/obstacle256_re100/{InputData,pattern.txt}

bench.py's reference arm runs the reference build on these directories, so it needs
nothing of this package at run time.  They are what mgfvm.configs.c1_pair(seed=1)
writes (a CPU test regenerates and compares them):

    python workloads/make_workloads.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "multigrid-fvm_b200"))

NAMES = ("obstacle256_re10", "obstacle256_re100")


def cases():
    from mgfvm import configs
    return dict(zip(NAMES, configs.c1_pair(seed=1)))


def main(out=HERE):
    for name, cfg in cases().items():
        cfg.write(os.path.join(out, name))
        print("wrote", os.path.join(out, name))


if __name__ == "__main__":
    main()
