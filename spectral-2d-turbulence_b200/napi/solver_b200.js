// solver_b200.js -- the reference's JavaScript Solver API (src/gpu/solver.js, lines 49-630)
// over the Node-API addon s2d_napi.c, which calls libs2d.so (hand-written sm_100a CUDA).
//
// Same class shape, method names, argument meaning and error behaviour as solver.js, so
// the reference's frame loop (src/main.js:389-467) and test harness hooks run against it:
//   - Solver.create(device, {n, dyeScale}) is async and resolves to a Solver; `device` is
//     the CUDA ordinal (a number) instead of a GPUDevice; the extra option `fft` selects
//     'fp32' (default), 'tc-f16' or 'tc-bf16';
//   - encode*(pass) / copyDiagnostics(encoder) accept and ignore the WebGPU pass /
//     encoder: work is enqueued on the solver's CUDA stream in call order;
//   - readDiagnostics() resolves to {spectrum, zonal, energy, enstrophy, dt, maxSpeed}
//     or null (nothing copied, a read already pending, destroyed, or a failed read);
//   - errors of the C ABI are thrown as Error with `code` = the negative status.
'use strict';

const path = require('path');

const addon = require(process.env.S2D_NAPI_ADDON ||
                      path.join(__dirname, 'build', 'Release', 's2d_napi.node'));

const MAX_SPLATS = 8;                                  // solver.js:9
const FFT = { fp32: 0, 'tc-f16': 1, 'tc-bf16': 2 };    // include/s2d.h S2D_FFT_*
const DYE = { none: 0, bands: 1 };                     // paintDye patterns (solver.js:446-473)
const BUF = {                                          // per-stage hook buffers (tests/index.html)
  state0: 0, state1: 1, state2: 2, packA: 3, packB: 4, physZ: 5, rhs: 6, force: 7, vel: 8, dt: 9,
};
const STEP = { dye: 1, reduce: 2, relatch: 4 };

function dyeCode(pattern) {
  if (!(pattern in DYE)) throw new Error(`unknown dye pattern ${pattern}`);
  return DYE[pattern];
}

class Solver {
  constructor(handle, n, dyeScale) {
    this.h = handle;
    this.n = n;
    this.ncells = n * n;
    this.m = n * dyeScale;
    this.nbins = n / 2 + 1;
    this.disposed = false;
    this.cfg = null;
  }

  static async create(device, { n = 256, dyeScale = 2, fft = 'fp32' } = {}) {
    if (!(fft in FFT)) throw new Error(`unknown fft path ${fft}`);
    const h = addon.create(n, dyeScale, FFT[fft], typeof device === 'number' ? device : 0);
    return new Solver(h, n, dyeScale);
  }

  // scalar state of solver.js:50-69, read from the library
  get phase() { return addon.info(this.h).phase; }
  get dyeParity() { return addon.info(this.h).dyeParity; }
  get stepIndex() { return addon.info(this.h).stepIndex; }
  get primed() { return addon.info(this.h).primed !== 0; }
  get simTime() { return addon.info(this.h).simTime; }
  set simTime(t) { addon.setSimTime(this.h, t); }
  get paramsF() {
    // the fields the reference's tests read (paramsF[2] is the mapped nuH, solver.js:311)
    const c = this.cfg || {};
    const info = addon.info(this.h);
    return Float32Array.from([c.beta ?? 0, c.drag ?? 0, info.nuH, c.hyperP ?? 0, c.forceAmp ?? 0,
      c.forceK ?? 0, c.forceWidth ?? 0, 0, (2 * Math.PI) / this.n, c.cfl ?? 0, c.dtMin ?? 0, c.dtMax ?? 0]);
  }

  configure(cfg) { addon.configure(this.h, cfg); this.cfg = cfg; }   // solver.js:306-324
  setSplats(list) { addon.setSplats(this.h, list || []); }          // solver.js:326-345

  seed({ k0 = 14, amplitude = 6, seed = 1 } = {}) {                  // solver.js:347-359
    addon.seed(this.h, k0, amplitude, seed >>> 0);
  }
  seedPhysical(values) {                                             // solver.js:361-382
    addon.seedPhysical(this.h, values instanceof Float32Array ? values : Float32Array.from(values));
  }
  reset(opts = {}) {                                                 // solver.js:420-444
    const field = opts.field ? (opts.field instanceof Float32Array ? opts.field : Float32Array.from(opts.field))
      : null;
    addon.reset(this.h, field, opts.k0 ?? 14, opts.amplitude ?? 6, (opts.seed ?? 1) >>> 0,
      dyeCode(opts.dyePattern ?? 'bands'));
  }
  paintDye(pattern) { addon.paintDye(this.h, dyeCode(pattern)); }   // solver.js:446-473

  encodePrime(_pass) { addon.encodePrime(this.h); }                  // solver.js:475-486
  encodeStep(_pass) { addon.encodeStep(this.h); }                    // solver.js:488-521
  encodeDye(_pass) { addon.encodeDye(this.h); }                      // solver.js:523-536
  encodeReduce(_pass) { addon.encodeReduce(this.h); }                // solver.js:538-545
  encodeDiagnostics(_pass) { addon.encodeDiagnostics(this.h); }      // solver.js:547-558
  copyDiagnostics(_encoder) { addon.copyDiagnostics(this.h); }       // solver.js:560-568

  async readDiagnostics() {                                          // solver.js:570-608
    if (this.disposed) return null;
    return addon.readDiagnostics(this.h);
  }

  // substeps of the main.js:413-419 loop in one call (optionally as a replayed CUDA graph)
  step(substeps = 1, { dye = true, reduce = true, graph = false, relatch = false } = {}) {
    const flags = (dye ? STEP.dye : 0) | (reduce ? STEP.reduce : 0) | (relatch ? STEP.relatch : 0);
    addon.step(this.h, substeps, flags, graph);
  }
  synchronize() { addon.synchronize(this.h); }

  // headless replacement of the dye texture (solver.js:610-612): binary16 rgba, M*M*4
  get currentDye() { return addon.currentDye(this.h); }

  // per-stage hooks of the reference's browser harness (tests/index.html:114-203)
  getBuffer(name) { return addon.getBuffer(this.h, BUF[name]); }
  setBuffer(name, values) {
    addon.setBuffer(this.h, BUF[name], values instanceof Float32Array ? values : Float32Array.from(values));
  }

  destroy() {                                                        // solver.js:614-629
    if (this.disposed) return;
    this.disposed = true;
    addon.destroy(this.h);
  }
}

// fft.js:20-31 and device.js:44-52 counterparts
function radixSchedule(n) { return addon.radixSchedule(n); }
function supportedGrids() { return addon.supportedGrids(); }

module.exports = { Solver, MAX_SPLATS, radixSchedule, supportedGrids, FFT, BUF };
