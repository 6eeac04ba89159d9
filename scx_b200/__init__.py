"""B200-native randomized PCA of sparse cells x genes matrices.

A from-scratch implementation of the scx-accel randomized PCA op
(``pyscx.accel.pca(..., device="gpu")``) on hand-written sm_100a kernels.
The compute lives in ``libscxpca.so`` (C ABI: ``include/scxpca.h``); this
package is the Python face of it.
"""

from .accel import PcaResult, Plan, gaussian, pca, randomized_pca, synth_nb_csr_device

__all__ = ["PcaResult", "Plan", "gaussian", "pca", "randomized_pca", "synth_nb_csr_device"]
__version__ = "0.1.0"
