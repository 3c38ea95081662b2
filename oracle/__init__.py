"""CPU oracle for the Plato Analyze linear-tet hot path.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use these modules to check (or time beside) the CUDA product.
The product library in platoanalyze_b200/ never imports or links anything here.

- np_ref.py : NumPy restatement for small meshes (golden-vector pinning).
- pa_oracle.cpp / cpu.py : FP64 C++/OpenMP restatement (same algorithm, any size).
"""
