"""B200-native grid kNN -> elliptic-Gabriel filter -> Taubin smoothing -> normals.

Host-side mirror of the reference's provider/consumer interface over the C-ABI
library built from multigpuegtsmoothing_b200/csrc.
"""
