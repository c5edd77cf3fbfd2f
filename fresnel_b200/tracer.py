"""Ray tracers (fresnel/tracer.py).

`Preview` renders a quick direct-lighting image; `Path` is the progressive Monte Carlo path
tracer.  Both keep their output on the device and copy it to the host when read.
"""

import numpy

from . import _common
from . import util

# numpy.histogram's bin edges for 512 bins over [0, 1] of float32 data (Tracer.histogram)
_HIST_EDGES = numpy.histogram(numpy.zeros(0, numpy.float32), bins=512, range=[0, 1])[1]


class Tracer:
    """Base class (fresnel/tracer.py:20-154)."""

    def __init__(self):
        raise RuntimeError("Use a specific tracer class")

    def resize(self, w, h):
        """Resize (and clear) the output buffer."""
        self._tracer.resize(w, h)

    def render(self, scene):
        """Render ``scene`` into the output buffer and return `output`."""
        self._tracer.render(scene._scene)
        return self.output

    def enable_highlight_warning(self, color=(1, 0, 1)):
        """Paint pixels brighter than 1 in any channel with ``color``."""
        self._tracer.enableHighlightWarning(_common.RGBf(*color))

    def disable_highlight_warning(self):
        self._tracer.disableHighlightWarning()

    def histogram(self):
        """Lightness and R, G, B histograms (512 bins, gamma 2.2) of the visible pixels
        (fresnel/tracer.py:79-108), computed on the device from the linear output (only the
        8 KB of counts cross to the host).  Returns ``(hist[512, 4] int64, bin_upper_edges)``;
        the edges are numpy.histogram's for 512 bins over [0, 1]."""
        counts = self._tracer.histogram()
        return counts.astype(numpy.int64), _HIST_EDGES[1:].copy()

    @property
    def output(self):
        """util.ImageArray: sRGB RGBA uint8 output (H, W, 4)."""
        return util.ImageArray(self._tracer.getSRGBOutputBuffer(), geom=None)

    @property
    def linear_output(self):
        """util.Array: linear RGBA float32 output (H, W, 4)."""
        return util.Array(self._tracer.getLinearOutputBuffer(), geom=None)

    @property
    def seed(self):
        return self._tracer.getSeed()

    @seed.setter
    def seed(self, value):
        self._tracer.setSeed(value)


class Preview(Tracer):
    """Direct-lighting preview tracer (fresnel/tracer.py:157-181).

    ``anti_alias=True`` takes 8 x 8 tent-filtered samples per pixel.
    """

    def __init__(self, device, w, h, anti_alias=True):
        self.device = device
        self._tracer = device.module.TracerDirect(device._device, w, h)
        self.anti_alias = anti_alias

    @property
    def anti_alias(self):
        return self._tracer.getAntialiasingN() > 1

    @anti_alias.setter
    def anti_alias(self, value):
        self._tracer.setAntialiasingN(8 if value else 1)


class Path(Tracer):
    """Progressive path tracer (fresnel/tracer.py:184-261).

    Each `render` adds one sample per pixel to the running mean.  `sample` takes many samples
    in one call; its result is identical to calling `render` that many times.
    """

    def __init__(self, device, w, h):
        self.device = device
        self._tracer = device.module.TracerPath(device._device, w, h, 1)

    def reset(self):
        """Clear the output and advance the seed (a statistically independent new image)."""
        self._tracer.reset()

    def sample(self, scene, samples, reset=True, light_samples=1):
        """Take ``samples`` samples per pixel, each with ``light_samples`` light paths."""
        if reset:
            self.reset()
        self._tracer.setLightSamples(light_samples)
        try:
            if samples > 0:
                self._tracer.renderSamples(scene._scene, samples)
        finally:
            # keep later render() calls at one light sample (fresnel/tracer.py:257-259)
            self._tracer.setLightSamples(1)
        return self.output


class PathBatch:
    """Path renders of many tracers and scenes traced together (no counterpart in fresnel).

    ``add(tracer, scene, samples, reset=True, light_samples=1)`` queues what
    ``tracer.sample(scene, samples, reset, light_samples)`` renders; ``render()`` traces every
    queued render in one CUDA graph launch. The renders share wavefronts, so many small frames
    keep the GPU as busy as one large frame. Afterwards each tracer holds the image its own
    ``sample`` call would have produced. Tracers and scenes can differ in size and content but
    must belong to the batch's device.
    """

    def __init__(self, device):
        self.device = device
        self._batch = device.module.Batch(device._device)
        self._queued = []

    def add(self, tracer, scene, samples, reset=True, light_samples=1):
        if tracer.device is not self.device or scene.device is not self.device:
            raise RuntimeError("Tracer, Scene and PathBatch devices do not match")
        if reset:
            if any(t is tracer for t in self._queued):
                raise RuntimeError("cannot reset a tracer that already has queued renders")
            tracer.reset()
        tracer._tracer.setLightSamples(light_samples)
        try:
            self._batch.add(tracer._tracer, scene._scene, samples)
        finally:
            tracer._tracer.setLightSamples(1)
        self._queued.append(tracer)

    def render(self):
        """Trace everything queued; the queue is empty afterwards."""
        try:
            self._batch.render()
        finally:
            self._queued = []

    def clear(self):
        self._batch.clear()
        self._queued = []

    def reserve(self, paths):
        """Allocate the path state for ``paths`` pixel samples in flight now, so that renders
        that fit allocate nothing (it grows on demand otherwise)."""
        self._batch.reserve(int(paths))

    def __len__(self):
        return len(self._batch)

    @property
    def stats(self):
        """Counters over the batch's lifetime: renders, waves, graph launches and captures,
        kernels run inside the graphs, device-side loop passes, traversal tests, device ms."""
        return self._batch.getStats()
