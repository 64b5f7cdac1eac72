"""Command line: clean one FITS image (``python -m cusmic_b200 SOURCE OUTPUT``).

A drop-in for the reference's FITS commands (``mod/cusmic/__main__.py``,
``src/main.c``): it accepts the same option names with the same defaults and
ranges, refuses to overwrite an existing output, needs ``--error`` or
``--gain`` when it detects, exits with 1 on a bad input and 2 on a usage
error.  The pixels are cleaned on the GPU by libcusmic_b200.so; FITS input and
output is ``cusmic_b200.fits``.
"""

from dataclasses import dataclass
from pathlib import Path

import click

from . import remove_cosmics
from .fits import read_fits, write_fits

_NONNEG = click.FloatRange(min=0)

# (flag, default, type, help): the detection settings, in the order the
# reference's commands list them.  Defaults are those of cusmic_default_options.
_SETTINGS = (
    ("--gain", None, click.FloatRange(min=0, min_open=True),
     "Detector gain (electrons per ADU) of the noise model; needed unless --error is given."),
    ("--readnoise", 0.0, _NONNEG, "Read noise (electrons) of the noise model."),
    ("--contrast", 3.0, _NONNEG, "Contrast of a cosmic ray over the fine-structure image."),
    ("--cr-threshold", 5.0, _NONNEG, "Significance (sigma) that seeds a cosmic ray."),
    ("--neighbor-threshold", 3.0, _NONNEG, "Significance (sigma) that grows a cosmic ray."),
    ("--maxiter", 4, click.IntRange(min=0), "Detection passes at most; 0 only copies the image."),
)


@dataclass(frozen=True)
class Job:
    """One cleaning as the command line asked for it."""
    source: Path
    output: Path
    error: Path = None
    gain: float = None
    readnoise: float = 0.0
    contrast: float = 3.0
    cr_threshold: float = 5.0
    neighbor_threshold: float = 3.0
    maxiter: int = 4

    def check(self):
        """Usage rules, before any file is read."""
        if self.output.name.startswith("!") or str(self.output).startswith("!"):
            # CFITSIO's "!" prefix would mean overwrite: not offered here.
            raise click.ClickException("Choose a new output filename")
        if self.output.exists():
            raise click.ClickException(f"{self.output} already exists; choose a new output")
        if self.maxiter > 0 and self.error is None and self.gain is None:
            raise click.UsageError("Provide --error or --gain (optionally --readnoise)")

    def run(self):
        """Read, clean on the GPU, write; returns the number of flagged pixels."""
        image, header = read_fits(self.source, dtype="float64")
        if image.ndim != 2:
            raise ValueError("The FITS command expects one 2D image")
        sigma = None if self.error is None else read_fits(self.error, dtype="float64")[0]
        cleaned, flagged = remove_cosmics(
            image, contrast=self.contrast, cr_threshold=self.cr_threshold,
            neighbor_threshold=self.neighbor_threshold, error=sigma,
            effective_gain=self.gain, readnoise=self.readnoise, maxiter=self.maxiter)
        flagged = flagged.cpu().numpy()
        header.add_history("cusmic_b200: cosmic rays removed (L.A.Cosmic)")
        write_fits(self.output, cleaned.cpu().numpy(), flagged, header=header)
        return int(flagged.sum())


def _command(func):
    """Attach the arguments and the settings table to the click command."""
    for flag, default, kind, text in reversed(_SETTINGS):
        func = click.option(flag, default=default, type=kind, help=text,
                            show_default=default is not None)(func)
    func = click.option("--error", type=click.Path(exists=True, dir_okay=False, path_type=Path),
                        help="FITS image of per-pixel 1-sigma errors (replaces the noise "
                             "model).")(func)
    func = click.argument("output", type=click.Path(dir_okay=False, path_type=Path))(func)
    func = click.argument("source",
                          type=click.Path(exists=True, dir_okay=False, path_type=Path))(func)
    return click.command()(func)


@_command
def main(source, output, **settings):
    """Clean SOURCE of cosmic rays and write the result to the new file OUTPUT
    (cleaned image in the primary HDU, the mask in a CRMASK extension)."""
    job = Job(source, output, **settings)
    job.check()
    try:
        count = job.run()
    except (OSError, ValueError, TypeError, IndexError, KeyError) as exc:
        raise click.ClickException(str(exc)) from exc
    click.echo(f"Saved {output} ({count:,} cosmic-ray pixels)")


if __name__ == "__main__":
    main()
