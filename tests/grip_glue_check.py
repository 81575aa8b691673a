"""Twin check for tests/test_gpu_gviz_adapter.py::test_grip_action_switch_bit_identical,
run in a fresh process (see that test): a GRIP state refined through the
"grip.refineRound" action after gvizCudaGripAttach (strict reductions) against
a twin refined by the reference on the CPU, every layer, then after detach.
Prints OK or the first mismatch."""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    from grapher_b200 import graphs
    from oracle.bindings import Reference
    ref = Reference()
    glue = C.CDLL(os.path.join(ROOT, "grapher_b200", "lib", "libgvizcuda_gviz.so"))
    glue.gvizCudaGripAttach.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    glue.gvizCudaGripDetach.argtypes = [C.c_void_p]
    glue.gvizCudaGripEmbedderLastError.argtypes = [C.c_void_p]
    a, b = graphs.barabasi_albert(600, 3, 5)
    cpu, gpu = ref.create_grip(600, a, b), ref.create_grip(600, a, b)
    cpu.begin()
    gpu.begin()
    g = C.c_void_p(gpu.state_ptr())
    if glue.gvizCudaGripAttach(g, 0, 1) != 0:
        return "attach failed"
    layers = 0
    while True:
        for r in range(4):
            cpu.refine()
            if gpu.invoke_refine() != 0 or glue.gvizCudaGripEmbedderLastError(g) != 0:
                return f"round failed at layer {cpu.layer}"
            if not np.array_equal(cpu.positions(), gpu.positions()):
                return f"positions differ at layer {cpu.layer} round {r}"
            (s1, r1), (s2, r2) = cpu.last_stats(), gpu.last_stats()
            if not (np.array_equal(s1, s2) and r1 == r2):
                return f"stats differ at layer {cpu.layer} round {r}"
        layers += 1
        if cpu.layer == 0:
            break
        cpu.next_stage()
        gpu.next_stage()
    if layers < 3:
        return f"only {layers} layers"
    glue.gvizCudaGripDetach(g)
    for r in range(3):
        cpu.refine()
        if gpu.invoke_refine() != 0 or not np.array_equal(cpu.positions(), gpu.positions()):
            return f"after detach round {r} differs"
    return "OK"


if __name__ == "__main__":
    print(main())
