"""Host-only helpers shared by tests, fixtures and the benchmark's CPU leg."""
from . import api


class HostSnelly(api.Snelly):
    """The scene-API facade without a GPU context: computes everything the host side uploads
    (scene options, uniform blocks, recorded scene uniforms) for use by CPU code."""

    def __init__(self, scene, seed=1):
        self._setup(scene, 256, 256, None)
        self.seed = seed
        self.initScene()

    def reset(self, no_recompile=False):
        self.pathtracer.numSamples = 0.0
        self.pathtracer.spp = 0.0
