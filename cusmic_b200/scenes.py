"""Seeded synthetic L.A.Cosmic scenes for benchmarks and large parity cases.

No public dataset is involved: each generator follows a written description of
a benchmark workload (sky level and noise, Gaussian stars, cosmic-ray hits and
tracks, bad-pixel masks, NaN holes) and draws everything from
``numpy.random.default_rng(seed)``.

Workloads:

* ``plain_512``: one 512 x 512 frame; sky 1000 ADU with Gaussian noise
  sigma = sqrt(1000*2 + 5^2)/2; 40 circular Gaussian stars (FWHM 2.5 px, peaks
  log-uniform in [200, 20000]); 150 cosmic rays (60% single pixels, 40%
  straight tracks 2-8 px at a uniform angle, amplitudes U[500, 15000]).
  Cleaned with gain=2, readnoise=5, contrast=3, cr=5, neighbor=3, maxiter=4.
* ``stack_2048``: 16 frames of 2048 x 2048 from the same generator, sky
  U[500, 3000] per frame, 400 stars and 1200 rays per frame; one shared error
  map sqrt(model/2 + 2.5^2) from frame 0's noiseless model; one shared mask with
  0.5% random bad pixels plus 2 full bad columns; 0.1% NaN pixels per frame.
* ``ragged_64``: 64 frames with heights and widths log-uniform in
  [256, 4096]; star and ray counts scaled by area from ``plain_512``; per-frame
  gain U[1, 4], readnoise U[2, 10], background U[0, 200].
* ``adjoint_1024``: 8 frames of 1024 x 1024 from ``plain_512``'s generator.
* ``large_8192``: 4 frames of 8192 x 8192; full-size error map; 2% random
  mask; 3000 rays per frame (10% long tracks of 10-40 px); 200 saturated stars
  clipped at 65535.
"""

from dataclasses import dataclass, field

import numpy as np

FWHM_TO_SIGMA = 1.0 / (2.0 * np.sqrt(2.0 * np.log(2.0)))


@dataclass
class Frame:
    data: np.ndarray
    model: np.ndarray
    gain: float = 2.0
    readnoise: float = 5.0
    background: float | None = 0.0


@dataclass
class Scene:
    name: str
    frames: list
    error: np.ndarray | None = None   # shared error map, if any
    mask: np.ndarray | None = None    # shared mask, if any
    settings: dict = field(default_factory=dict)

    @property
    def pixels(self):
        return sum(f.data.size for f in self.frames)


def _stars(rng, model, count, peak_lo, peak_hi, fwhm=2.5, clip=None):
    h, w = model.shape
    sigma = fwhm * FWHM_TO_SIGMA
    rad = int(np.ceil(6 * sigma))
    ys = rng.uniform(0, h, count)
    xs = rng.uniform(0, w, count)
    peaks = np.exp(rng.uniform(np.log(peak_lo), np.log(peak_hi), count))
    oy, ox = np.mgrid[-rad:rad + 1, -rad:rad + 1]
    for y, x, p in zip(ys, xs, peaks):
        cy, cx = int(y), int(x)
        yy, xx = oy + cy, ox + cx
        ok = (yy >= 0) & (yy < h) & (xx >= 0) & (xx < w)
        r2 = (yy - y) ** 2 + (xx - x) ** 2
        model[yy[ok], xx[ok]] += p * np.exp(-0.5 * r2[ok] / sigma ** 2)
    if clip is not None:
        np.minimum(model, clip, out=model)


def _rays(rng, data, count, track_frac, len_lo, len_hi, amp_lo=500.0, amp_hi=15000.0):
    h, w = data.shape
    ys = rng.integers(0, h, count)
    xs = rng.integers(0, w, count)
    amps = rng.uniform(amp_lo, amp_hi, count)
    tracks = rng.random(count) < track_frac
    lengths = rng.uniform(len_lo, len_hi, count)
    angles = rng.uniform(0, np.pi, count)
    for y, x, a, t, ln, ang in zip(ys, xs, amps, tracks, lengths, angles):
        if not t:
            data[y, x] += a
            continue
        steps = max(2, int(np.ceil(ln * 2)))
        s = np.linspace(-ln / 2, ln / 2, steps)
        py = np.clip(np.rint(y + s * np.sin(ang)).astype(int), 0, h - 1)
        px = np.clip(np.rint(x + s * np.cos(ang)).astype(int), 0, w - 1)
        cells = np.unique(py * w + px)
        data.flat[cells] += a


def make_frame(rng, h, w, *, sky=1000.0, n_stars=40, n_rays=150, gain=2.0, readnoise=5.0,
               track_frac=0.4, len_lo=2.0, len_hi=8.0, peak_lo=200.0, peak_hi=20000.0,
               clip=None, background=0.0):
    model = np.full((h, w), sky, dtype=np.float64)
    _stars(rng, model, n_stars, peak_lo, peak_hi, clip=clip)
    sigma = np.sqrt(sky * gain + readnoise ** 2) / gain
    data = model + rng.normal(0.0, sigma, (h, w))
    _rays(rng, data, n_rays, track_frac, len_lo, len_hi)
    if clip is not None:
        np.minimum(data, clip, out=data)
    return Frame(data, model, gain, readnoise, background)


PLAIN = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4,
             border="mirror")


def plain_512(seed=0, size=512):
    rng = np.random.default_rng(seed)
    f = make_frame(rng, size, size)
    return Scene("plain_512", [f], settings=dict(PLAIN))


def stack_2048(seed=0, frames=16, size=2048):
    rng = np.random.default_rng(seed)
    area = (size * size) / (2048 * 2048)
    out = []
    for _ in range(frames):
        sky = rng.uniform(500, 3000)
        out.append(make_frame(rng, size, size, sky=sky, n_stars=max(1, int(400 * area)),
                              n_rays=max(1, int(1200 * area)), background=None))
    error = np.sqrt(out[0].model / 2 + 2.5 ** 2)
    mask = rng.random((size, size)) < 0.005
    cols = rng.choice(size, 2, replace=False)
    mask[:, cols] = True
    for f in out:
        nan = rng.random((size, size)) < 0.001
        f.data[nan] = np.nan
    return Scene("stack_2048", out, error=error, mask=mask,
                 settings=dict(PLAIN, maxiter=4))


def ragged_shapes(seed=0, frames=64, lo=256, hi=4096):
    rng = np.random.default_rng(seed)
    hs = np.exp(rng.uniform(np.log(lo), np.log(hi), frames)).astype(int)
    ws = np.exp(rng.uniform(np.log(lo), np.log(hi), frames)).astype(int)
    return list(zip(hs.tolist(), ws.tolist())), rng


def ragged_64(seed=0, frames=64, lo=256, hi=4096):
    shapes, rng = ragged_shapes(seed, frames, lo, hi)
    out = []
    for h, w in shapes:
        area = h * w / 512 ** 2
        gain, rn, bg = rng.uniform(1, 4), rng.uniform(2, 10), rng.uniform(0, 200)
        f = make_frame(rng, h, w, n_stars=max(1, int(round(40 * area))),
                       n_rays=max(1, int(round(150 * area))), gain=gain, readnoise=rn,
                       background=bg)
        out.append(f)
    return Scene("ragged_64", out, settings=dict(PLAIN))


def adjoint_1024(seed=0, frames=8, size=1024):
    rng = np.random.default_rng(seed)
    area = size * size / 512 ** 2
    out = [make_frame(rng, size, size, n_stars=int(40 * area), n_rays=int(150 * area))
           for _ in range(frames)]
    return Scene("adjoint_1024", out, settings=dict(PLAIN))


def large_8192(seed=0, frames=4, size=8192):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(frames):
        out.append(make_frame(rng, size, size, n_stars=200, n_rays=0, clip=65535.0,
                              peak_lo=20000.0, peak_hi=200000.0, background=None))
        f = out[-1]
        _rays(rng, f.data, 2700, 0.0, 1, 1)
        _rays(rng, f.data, 300, 1.0, 10.0, 40.0)
        np.minimum(f.data, 65535.0, out=f.data)
    error = np.sqrt(out[0].model / 2 + 2.5 ** 2)
    mask = rng.random((size, size)) < 0.02
    return Scene("large_8192", out, error=error, mask=mask, settings=dict(PLAIN))


WORKLOADS = {
    "plain_512": plain_512,
    "stack_2048": stack_2048,
    "ragged_64": ragged_64,
    "adjoint_1024": adjoint_1024,
    "large_8192": large_8192,
}
