"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs in a container that has the reference sources (it uses oracle/_ref/
libref_cpu.so, built from Kernel/cuda/src/Matrix.h by oracle/build_ref.py):
  * inputs from Matrix<T>::fillRandom(seed)   (Matrix.h:75-87: mt19937(seed), U[0,1))
  * products from Matrix<double>::operator*    (Matrix.h:183-201) and
    Matrix<float>::operator* (accumulating in float, the reference's own CPU path)
Each fixture stores A, B (float32 as the reference draws them), the FP64
product and the FP32 product.  Re-run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# (m, n, k, seedA, seedB): small odd shapes of the reference's square / special families
SHAPES = [(1, 1, 1, 0, 1), (7, 5, 3, 0, 1), (16, 24, 40, 0, 1), (33, 17, 65, 2, 3), (64, 64, 64, 0, 0),
          (127, 9, 31, 4, 5), (4, 8, 300, 6, 7)]


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libref_cpu.so missing: run python oracle/build_ref.py first")
    for m, n, k, sa, sb in SHAPES:
        A = oracle.ref_fill_random(sa, m, k, np.float32)
        B = oracle.ref_fill_random(sb, k, n, np.float32)
        p64 = oracle.ref_product(A, B)
        p32 = np.empty((m, n), np.float32)
        import ctypes as C

        oracle.ref_cpu().ref_cpu_gemm_f32(m, n, k, A.ctypes.data_as(C.POINTER(C.c_float)),
                                          B.ctypes.data_as(C.POINTER(C.c_float)),
                                          p32.ctypes.data_as(C.POINTER(C.c_float)))
        np.savez_compressed(os.path.join(HERE, "gemm_%dx%dx%d.npz" % (m, n, k)), A=A, B=B, prod_f64=p64,
                            prod_f32=p32, seeds=np.array([sa, sb]))
    print("wrote", len(SHAPES), "fixtures")


if __name__ == "__main__":
    main()
