"""Headless pointer strokes (src/ui/pointer.js) -> splat lists; host logic, no GPU."""
import math


def test_stroke_produces_splats(pkg):
    p = pkg.Pointer()
    p.onMove(0.5, 0.5)                      # not pressed: ignored
    p.onDown(0.2, 0.3)
    p.onMove(0.2, 0.3)                      # no motion: ignored (pointer.js:56-58)
    p.onMove(0.25, 0.31)
    p.onMove(0.3, 0.35)
    p.onUp()
    p.onMove(0.9, 0.9)                      # released: ignored
    out = p.collect()
    assert len(out) == 2
    a = out[0]
    assert (a["x"], a["y"]) == (0.25, 0.31)
    assert math.isclose(a["dx"], 0.05) and math.isclose(a["dy"], 0.01)
    assert a["color"] == pkg.pointer.PALETTE[1]          # stroke advanced on pointerdown
    assert a["radius"] == 0.045 and a["amp"] == 400
    assert math.isclose(a["dyeAmp"], min(1.0, math.hypot(0.05, 0.01) * 40))
    assert p.collect() == []


def test_pending_is_capped_and_palette_cycles(pkg):
    p = pkg.Pointer()
    for stroke in range(7):
        p.onDown(0.0, 0.0)
        for k in range(1, 4):
            p.onMove(0.01 * k, 0.0)
        p.onUp()
    out = p.collect()
    assert len(out) == pkg.MAX_SPLATS                    # pointer.js:60
    assert p.stroke == 7 % len(pkg.pointer.PALETTE)
    loc = pkg.Pointer.locate(150, 50, 100, 0, 200, 100)
    assert loc == {"x": 0.25, "y": 0.5}


def test_splats_feed_setsplats_shape(pkg):
    p = pkg.Pointer(radius=0.05, strength=300, dyeAmount=0.5)
    p.onDown(0.5, 0.5)
    p.onMove(0.52, 0.5)
    (sp,) = p.collect()
    assert set(sp) == {"x", "y", "dx", "dy", "color", "radius", "amp", "dyeAmp"}   # solver.js:326-345 keys
