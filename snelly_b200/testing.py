"""Host-only helpers shared by tests, fixtures and the benchmark's CPU leg."""
from . import api


class HostSnelly(api.Snelly):
    """The scene-API facade without a GPU context: computes everything the host side uploads
    (scene options, uniform blocks, recorded scene uniforms) for use by CPU code."""

    def __init__(self, scene, seed=1):
        self.sceneObj = scene
        self.width = self.height = 256
        self.camera = api.Camera()
        self.camControls = api.Controls()
        self.materials = api.Materials()
        self.pathtracer = api.Renderer(self)
        self.spectra = {}
        self.spectrumObj = None
        self._job = None
        self._ctx = None
        self._scene_key = None
        self.seed = seed
        self.initScene()

    def reset(self, no_recompile=False):
        self.pathtracer.spp = 0.0
