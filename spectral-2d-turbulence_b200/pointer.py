"""Headless pointer input (src/ui/pointer.js): strokes in normalised coordinates become
the splat list ``Solver.setSplats`` takes.

The reference reads pointer events from a canvas and maps them with ``locate``
(pointer.js:34-40: x = (clientX - left)/width, y = 1 - (clientY - top)/height); here
the caller passes those normalised positions directly (there is no canvas).
"""
from __future__ import annotations

import math

from .solver import MAX_SPLATS

PALETTE = [                                       # pointer.js:3-10
    (1.0, 0.42, 0.28),
    (0.34, 0.78, 1.0),
    (1.0, 0.82, 0.32),
    (0.62, 0.48, 1.0),
    (0.36, 0.93, 0.66),
    (1.0, 0.5, 0.78),
]


class Pointer:
    """pointer.js:12-81 without the DOM: ``onDown(x, y)``, ``onMove(x, y)``, ``onUp()``,
    ``collect()``."""

    def __init__(self, radius: float = 0.045, strength: float = 400.0, dyeAmount: float = 1.0):
        self.pending = []
        self.active = False
        self.last = None
        self.stroke = 0
        self.radius = radius
        self.strength = strength
        self.dyeAmount = dyeAmount

    @staticmethod
    def locate(client_x, client_y, left, top, width, height):
        """pointer.js:34-40: canvas-relative position, y up."""
        return {"x": (client_x - left) / width, "y": 1 - (client_y - top) / height}

    def onDown(self, x: float, y: float):                   # pointer.js:42-47
        self.active = True
        self.stroke = (self.stroke + 1) % len(PALETTE)
        self.last = {"x": x, "y": y}

    def onMove(self, x: float, y: float):                   # pointer.js:49-71
        if not self.active:
            return
        dx = x - self.last["x"]
        dy = y - self.last["y"]
        self.last = {"x": x, "y": y}
        if dx == 0 and dy == 0:
            return
        if len(self.pending) < MAX_SPLATS:
            self.pending.append({
                "x": x, "y": y, "dx": dx, "dy": dy, "color": PALETTE[self.stroke],
                "radius": self.radius, "amp": self.strength,
                "dyeAmp": self.dyeAmount * min(1.0, math.hypot(dx, dy) * 40),
            })

    def onUp(self):                                         # pointer.js:73-76
        self.active = False
        self.last = None

    def collect(self):                                      # pointer.js:78-82
        out, self.pending = self.pending, []
        return out
