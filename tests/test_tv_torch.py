"""The differentiable TV-SQS terms (torch ops) against the FP64 oracle, on CPU.
Weights and eps are exact in float32, as the oracle rounds them like the kernel."""
import numpy as np

from conftest import rel_l2


def test_tv_torch_matches_oracle_on_cpu(oracle):
    import torch

    from ctprojector_b200.autograd import tv_sqs_torch

    rng = np.random.default_rng(9)
    img = rng.uniform(0, 1, (2, 3, 11, 13))
    ours = tv_sqs_torch(torch.tensor(img), (0.25, 1.0, 2.0), 2.0 ** -26)
    ref = oracle.tv_sqs(img, (0.25, 1.0, 2.0), 2.0 ** -26)
    for a, b in zip(ours, ref):
        assert rel_l2(a.numpy(), b) <= 1e-12
