"""A thin torch.autograd.Function over the library's forward solve and adjoint gradient (test harness
only): vertices (nv x 3, float64, CPU) -> (D_t, D_r, CHI'), backward through bgpu_best_gradient."""
import numpy as np
import torch

import best_hydro_b200 as bh
from best_hydro_b200 import meshes


class BestValues(torch.autograd.Function):
    @staticmethod
    def forward(ctx, verts, faces, truearea, iarea):
        v = verts.detach().cpu().numpy()
        st = bh.Setup(meshes.to_triangles(v, faces), iarea, truearea)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        xmu, gdef = st.deflation(s.diag_mean())
        bh.set_precision(bh.BGPU_FP64)
        s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        vals, g = s.gradient(iarea=iarea, truearea=truearea or 0.0)
        bh.set_precision(-1)
        ctx.save_for_backward(torch.from_numpy(meshes.corner_to_vertex(g, faces, len(v))))
        return torch.from_numpy(vals)

    @staticmethod
    def backward(ctx, gout):
        (gv,) = ctx.saved_tensors  # (3 results, nv, 3)
        return torch.einsum("k,kvc->vc", gout, gv), None, None, None
