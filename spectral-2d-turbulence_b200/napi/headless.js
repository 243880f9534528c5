// headless.js -- the reference's frame loop (src/main.js:389-467) without the renderer,
// driving solver_b200.js:
//
//   node headless.js [--n 1024] [--dye-scale 2] [--fft fp32|tc-f16|tc-bf16] [--frames 600]
//                    [--substeps 1] [--device 0]
//
// Per frame, in the reference's order: configure(config) and setSplats(pointer splats),
// encodePrime once, `substeps` x (encodeStep, encodeDye, encodeReduce), every 6th frame
// encodeDiagnostics + copyDiagnostics and an async readDiagnostics whose result is kept
// when it resolves (while later frames run); simTime advances by the last diagnostics dt.
// Pointer strokes are synthetic: a circle traced at the frame rate, turned into splats the
// way ui/pointer.js:46-80 does.  Prints one stats line every 60 frames.
'use strict';

const { Solver } = require('./solver_b200.js');

function parseArgs(argv) {
  const a = { n: 1024, dyeScale: 2, fft: 'fp32', frames: 600, substeps: 1, device: 0 };
  for (let i = 0; i < argv.length; i += 2) {
    const k = argv[i].replace(/^--/, '');
    const v = argv[i + 1];
    if (k === 'n') a.n = parseInt(v, 10);
    else if (k === 'dye-scale') a.dyeScale = parseInt(v, 10);
    else if (k === 'fft') a.fft = v;
    else if (k === 'frames') a.frames = parseInt(v, 10);
    else if (k === 'substeps') a.substeps = parseInt(v, 10);
    else if (k === 'device') a.device = parseInt(v, 10);
    else throw new Error(`unknown option --${k}`);
  }
  return a;
}

// the main.js config keys the step reads (values of its 'inverse cascade' preset style)
const config = {
  beta: 0, drag: 0.01, viscosity: 1.0, hyperP: 4, forceAmp: 0.1, forceK: 64, forceWidth: 2,
  cfl: 0.5, dtMin: 1e-6, dtMax: 1e-3, dyeFade: 0.999, paused: false, stirStrength: 1.0, stirRadius: 0.03,
};

// a stroke along a circle: splats from consecutive positions (pointer.js:46-80 shape)
function strokeSplats(frame, strength, radius) {
  const t0 = frame * 0.02, t1 = (frame + 1) * 0.02;
  const p0 = [0.5 + 0.25 * Math.cos(t0), 0.5 + 0.25 * Math.sin(t0)];
  const p1 = [0.5 + 0.25 * Math.cos(t1), 0.5 + 0.25 * Math.sin(t1)];
  const hue = (frame % 360) / 360;
  const color = [0.5 + 0.5 * Math.cos(2 * Math.PI * hue), 0.5 + 0.5 * Math.cos(2 * Math.PI * (hue + 1 / 3)),
    0.5 + 0.5 * Math.cos(2 * Math.PI * (hue + 2 / 3))];
  return [{ x: p1[0], y: p1[1], dx: (p1[0] - p0[0]) * 60, dy: (p1[1] - p0[1]) * 60, color, radius,
    amp: strength, dyeAmp: 1.0 }];
}

async function main() {
  const args = parseArgs(process.argv.slice(2));
  const solver = await Solver.create(args.device, { n: args.n, dyeScale: args.dyeScale, fft: args.fft });
  solver.configure(config);
  solver.reset({ k0: 14, amplitude: 6, seed: 1, dyePattern: 'bands' });
  let diagnostics = null;
  const t0 = process.hrtime.bigint();
  for (let tick = 0; tick < args.frames; tick += 1) {
    solver.configure(config);
    solver.setSplats(config.paused ? [] : strokeSplats(tick, config.stirStrength, config.stirRadius));
    const wantDiagnostics = tick % 6 === 0;
    if (!solver.primed) solver.encodePrime();
    if (!config.paused) {
      for (let i = 0; i < args.substeps; i += 1) {
        solver.encodeStep();
        solver.encodeDye();
        solver.encodeReduce();
      }
    }
    if (wantDiagnostics) {
      solver.encodeDiagnostics();
      solver.copyDiagnostics();
      solver.readDiagnostics().then((r) => { if (r) diagnostics = r; }).catch(() => {});
    }
    if (diagnostics && !config.paused) solver.simTime += diagnostics.dt * args.substeps;
    if (tick % 60 === 59) {
      await new Promise((r) => setImmediate(r));   // let pending reads resolve
      const secs = Number(process.hrtime.bigint() - t0) / 1e9;
      const d = diagnostics;
      console.log([`frame ${tick + 1}`, `${((tick + 1) / secs).toFixed(0)} fps`,
        d ? `dt ${d.dt.toExponential(2)}` : 'dt -', d ? `u_max ${d.maxSpeed.toFixed(2)}` : 'u_max -',
        d ? `E ${d.energy.toFixed(4)}` : 'E -', d ? `Z ${d.enstrophy.toFixed(2)}` : 'Z -',
        `t ${solver.simTime.toFixed(3)}`].join('   '));
    }
  }
  solver.synchronize();
  solver.destroy();
}

main().catch((e) => { console.error(e); process.exit(1); });
