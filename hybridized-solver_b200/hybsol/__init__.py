"""hybsol on a B200: the hybridized solver's block-sparse LU, factored on the GPU.

Drop-in for the reference package's public surface: ``hybsol.BlockSystem`` (the
``hybsol._mod`` extension type) and the helpers of ``hybsol.system``.
"""

from hybsol.system import BlockSystem as BlockSystem
