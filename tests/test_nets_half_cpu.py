"""Nets declared `half` compile to a tensor-core stage kernel (tcgen05) for sm_100a, without a GPU; a net without
`half` keeps the fp32 per-cell form."""
import os

from conftest import ROOT
from test_nets_half_gpu import half


def test_half_nets_generate_tensor_core_stages(monkeypatch):
    from fieldcuda.solver import compile_check, cuda_source
    monkeypatch.chdir(ROOT)
    for law in ("nets_mlp.law", "nets_flux.law", "nets_ldiffuse.law"):
        text = open(os.path.join(ROOT, "tests", "laws", law)).read()
        src = cuda_source(half(text), 20, 14, 9, 0.5)
        assert "fe_net_pass<" in src and "tcgen05.mma.cta_group::1.kind::f16" in src, law
        assert "fe_net_pass<" not in cuda_source(text, 20, 14, 9, 0.5).split("#endif // FE_DEVICE_CUH")[-1], law
        compile_check(half(text), 20, 14, 9, 0.5)
