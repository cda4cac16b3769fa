"""Minimal column logger with the interface the solver uses
(``pr`` and ``st``, ContactMechanics/Tools/Logger.py:102-233).

A solver given a logger other than ``quiet`` reports every iteration that
did not converge through the library's per-iteration observer, then the
final ``force_print=True`` line (ConstrainedConjugateGradients.py:436-495).
"""
import sys


class Logger(object):
    def __init__(self, logfile=sys.stdout, outevery=1, sepevery=10):
        self.logfile = logfile
        self.outevery = outevery
        self.sepevery = sepevery

    def _print(self, s):
        if self.logfile is None:
            return
        if isinstance(self.logfile, str):
            with open(self.logfile, "a") as fh:
                print(s, file=fh)
        else:
            print(s, file=self.logfile)

    def pr(self, s, caller=None, logfile=None):
        self._print(s)

    def warn(self, s, caller=None):
        self.pr("Warning: " + s)

    def st(self, hdr, vals, force_print=False):
        assert len(hdr) == len(vals)
        self._print("#" + "  ".join("{}:{}".format(i + 1, h) for i, h in enumerate(hdr)))
        self._print(" " + "  ".join(
            "{:>20.12e}".format(v) if isinstance(v, float) else "{:>20}".format(str(v))
            for v in vals))


quiet = Logger(None)
screen = Logger()
