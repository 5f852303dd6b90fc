"""Minimal logger with the reference's section/dump/set_level interface
(cmmdft/log.py:45-289): sections accumulate wall time per timer label."""
import sys
import time
from contextlib import contextmanager

__all__ = ['log']


class Logger(object):
    def __init__(self):
        self.log_level = 1
        self.timetable = {}
        self.warnings = []

    def set_level(self, level):
        if isinstance(level, str):
            level = ['silent', 'low', 'medium', 'high'].index(level.lower())
        self.log_level = level

    @contextmanager
    def section(self, label, level, timer=None):
        t0 = time.perf_counter()
        try:
            yield
        finally:
            if timer is not None:
                self.timetable[timer] = self.timetable.get(timer, 0.0) + time.perf_counter() - t0

    def dump(self, message, level=2):
        if self.log_level >= level:
            print(message, file=sys.stdout)

    def warning(self, message, label_section=None):
        self.warnings.append(message)


log = Logger()
