"""bench.py's bookkeeping on CPU: the kernel list follows the launch choices,
the roofline traffic is keyed by that list, and the ANN's tensor-core work
uses each model's descriptor length (NEP4: n_R + n_A (l_max + 4-body +
5-body))."""
import bench


class FakePot:
    def __init__(self, fused):
        self.fused = fused

    def tuning(self):
        return {"fused_f12": self.fused}, True


def test_force_kernels_follow_the_angular_force_form():
    assert bench.force_kernels(FakePot(1)) == ["k_filter_radial", "k_nep_fused", "k_gather"]
    assert bench.force_kernels(FakePot(0)) == ["k_filter_radial", "k_nep_fused", "k_angular_f12",
                                               "k_gather"]


def test_traffic_is_keyed_by_the_captured_kernel_list():
    key = ("carbon8m", tuple(bench.force_kernels(FakePot(1))))
    assert key in bench.TRAFFIC_PER_ATOM
    assert 3000 < bench.TRAFFIC_PER_ATOM[key] < 4000   # bytes per atom and force call
    assert ("carbon8m", tuple(bench.force_kernels(FakePot(0)))) not in bench.TRAFFIC_PER_ATOM


def test_ann_tensor_work_uses_the_descriptor_length():
    carbon = bench.ann_tensor_fraction({"spec": bench.WORKLOADS["carbon8m"]}, 1.0e8)
    assert (carbon["dim"], carbon["H"]) == (35, 30)           # l_max 4 2 1: 5 + 5 * 6
    assert carbon["flops_per_atom"] == 4 * 35 * 30
    water = bench.ann_tensor_fraction({"spec": bench.WORKLOADS["water"]}, 1.0e8)
    assert (water["dim"], water["H"]) == (30, 50)             # l_max 4 2 0: 5 + 5 * 5
    assert abs(water["achieved_tflops"] - 1.0e8 * 6000 / 1e12) < 1e-12
