/**
 * StepLoop over libmdb200 -- the TypeScript surface of src/gpu/loop.ts,
 * backed by the B200 engine through the Node-API addon in ../napi/addon.cc.
 *
 * Same public members, same units, same named errors as the reference's
 * `StepLoop` (src/gpu/loop.ts:208-1116), so `LoopEngine` (src/gpu/engine.ts)
 * and `runProtocol` (src/engine/protocol.ts) can take it unchanged.  Every call
 * is synchronous in the addon; the Promises resolve after it returns.
 *
 * Not verified on this machine: there is no Node runtime and no node_api.h
 * here or on the GPU box.  The Python mirror (mdb200/steploop.py) exercises
 * the same C ABI in the tests.
 */

import { parseState } from "../../src/engine/state.js";
import type { OpenMMState } from "../../src/engine/state.js";
import { parseSystem } from "../../src/engine/system.js";
import type { OpenMMSystem } from "../../src/engine/system.js";
import type { PoolReport } from "../../src/gpu/allocator.js";
import type { RunOptions, Report } from "../../src/gpu/loop.js";
import { kineticEnergy, shiftedKineticEnergy } from "../../src/reference/kinetic.js";

// eslint-disable-next-line @typescript-eslint/no-require-imports
const addon = require("./build/Release/mdb200.node") as MdbAddon;

type Vec3 = [number, number, number];

interface Energies {
  readonly potential: number;
  readonly kinetic: number;
  readonly temperature: number;
  readonly directGroup: number;
  readonly reciprocalGroup: number;
  readonly [group: string]: number;
}

interface MdbAddon {
  create(system: OpenMMSystem, state: OpenMMState, options: RunOptions): unknown;
  run(handle: unknown, steps: number): void;
  evaluate(handle: unknown, forces: Float64Array | null): Energies;
  potential(handle: unknown, positions: Float64Array, forces: Float64Array): Energies;
  positions(handle: unknown, out: Float64Array): void;
  velocities(handle: unknown, out: Float64Array): void;
  setPositions(handle: unknown, positions: Float64Array): void;
  setVelocities(handle: unknown, velocities: Float64Array): void;
  setBox(handle: unknown, vectors: Float64Array): void;
  box(handle: unknown): Float64Array;
  mesh(handle: unknown): Int32Array;
  setStep(handle: unknown, step: number): void;
  step(handle: unknown): number;
  barostat(handle: unknown): { attempts: number; accepted: number; volumeScale: number };
  neighbours(handle: unknown): {
    rebuilds: number;
    tiles: number;
    overflowed: boolean;
    capacity: number;
    skin: number;
    byteLength: number;
    innerTiles: number;
    prunes: number;
  };
  cellGeometry(handle: unknown): { divisions: number[]; extent: number[] };
  passesPerStep(handle: unknown): number;
  memory(handle: unknown): { count: number; totalBytes: number };
  destroy(handle: unknown): { leaked: number };
}

export class StepLoop {
  private constructor(
    private readonly handle: unknown,
    private readonly system: OpenMMSystem,
    readonly options: RunOptions,
  ) {}

  /** `StepLoop.create`, loop.ts:268: parse the System and State XML, then `fromParsed`. */
  static async create(
    device: unknown,
    texts: { readonly systemXml: string; readonly stateXml: string },
    options: RunOptions,
  ): Promise<StepLoop> {
    return StepLoop.fromParsed(device, parseSystem(texts.systemXml), parseState(texts.stateXml), options);
  }

  /** `StepLoop.fromParsed`, loop.ts:278.  The GPU device is chosen by `options`. */
  static async fromParsed(
    _device: unknown,
    system: OpenMMSystem,
    state: OpenMMState,
    options: RunOptions,
  ): Promise<StepLoop> {
    return new StepLoop(addon.create(system, state, options), system, options);
  }

  get steps(): number {
    return addon.step(this.handle);
  }

  advanceStepCount(step: number): void {
    if (!Number.isInteger(step) || step < 0) {
      throw new Error(`a step count must be a non-negative integer, got ${step}`);
    }
    addon.setStep(this.handle, step);
  }

  /** `StepLoop.run(n)`, loop.ts:651 -- barostat attempts included. */
  async run(steps: number): Promise<void> {
    if (steps > 0) addon.run(this.handle, steps);
  }

  /** `StepLoop.evaluateForces`, loop.ts:924: one force evaluation at the current coordinates, no step. */
  async evaluateForces(): Promise<void> {
    addon.evaluate(this.handle, null);
  }

  /**
   * `StepLoop.report`, loop.ts:761: the potential at the current coordinates,
   * the kinetic energy as the velocities stand, and the shifted kinetic energy
   * (velocities advanced half a step and re-constrained) through the
   * reference's own host function, as its report computes it.
   */
  async report(): Promise<Report> {
    const forces = new Float64Array(this.system.particleCount * 3);
    const e = addon.evaluate(this.handle, forces);
    const positions = await this.positions();
    const velocities = await this.velocities();
    const unshifted = kineticEnergy(this.system, velocities);
    const shifted = shiftedKineticEnergy(this.system, positions, velocities, forces, 0.5 * this.options.timeStep);
    const step = this.steps;
    return {
      step,
      time: step * this.options.timeStep,
      potentialEnergy: e.potential,
      kineticEnergy: unshifted,
      shiftedKineticEnergy: shifted,
      totalEnergy: e.potential + shifted,
      temperature: e.temperature,
    };
  }

  async potential(positions: Float64Array): Promise<{ energy: number; forces: Float64Array }> {
    const forces = new Float64Array(this.system.particleCount * 3);
    const e = addon.potential(this.handle, positions, forces);
    return { energy: e.potential, forces };
  }

  async positions(): Promise<Float64Array> {
    const out = new Float64Array(this.system.particleCount * 3);
    addon.positions(this.handle, out);
    return out;
  }

  async velocities(): Promise<Float64Array> {
    const out = new Float64Array(this.system.particleCount * 3);
    addon.velocities(this.handle, out);
    return out;
  }

  setPositions(positions: Float64Array): void {
    if (positions.length !== this.system.particleCount * 3) {
      throw new Error(`expected ${this.system.particleCount * 3} coordinates, got ${positions.length}`);
    }
    addon.setPositions(this.handle, positions);
  }

  setVelocities(velocities: Float64Array): void {
    if (velocities.length !== this.system.particleCount * 3) {
      throw new Error(`expected ${this.system.particleCount * 3} velocities, got ${velocities.length}`);
    }
    addon.setVelocities(this.handle, velocities);
  }

  setBox(vectors: readonly [Vec3, Vec3, Vec3]): void {
    addon.setBox(this.handle, Float64Array.from(vectors.flat()));
  }

  get mesh(): Vec3 {
    const m = addon.mesh(this.handle);
    return [m[0] as number, m[1] as number, m[2] as number];
  }

  /** `StepLoop.boxLengths`, loop.ts:995: the box's diagonal (its product is the volume). */
  get boxLengths(): Vec3 {
    const b = this.boxVectorsNow;
    return [b[0][0], b[1][1], b[2][2]];
  }

  get boxVectorsNow(): [Vec3, Vec3, Vec3] {
    const b = addon.box(this.handle);
    return [
      [b[0] as number, b[1] as number, b[2] as number],
      [b[3] as number, b[4] as number, b[5] as number],
      [b[6] as number, b[7] as number, b[8] as number],
    ];
  }

  /** `StepLoop.barostatStatistics`, loop.ts:572: null when the System has no MonteCarloBarostat. */
  get barostatStatistics(): { attempts: number; accepted: number; volumeScale: number } | null {
    if (!this.system.forces.some((f) => f.type === "MonteCarloBarostat")) return null;
    return addon.barostat(this.handle);
  }

  /**
   * `StepLoop.verletFlags`, loop.ts:941.  `worstDisplacement` is NaN: the
   * engine tests each atom's displacement against half the skin on the device
   * and keeps no maximum.  `capacity` counts cluster-pair tiles.
   */
  async verletFlags(): Promise<{
    readonly rebuilds: number;
    readonly worstDisplacement: number;
    readonly overflowed: boolean;
    readonly capacity: number;
    readonly skin: number;
    readonly byteLength: number;
  }> {
    const n = addon.neighbours(this.handle);
    return {
      rebuilds: n.rebuilds,
      worstDisplacement: Number.NaN,
      overflowed: n.overflowed,
      capacity: n.capacity,
      skin: n.skin,
      byteLength: n.byteLength,
    };
  }

  /** `StepLoop.cellGeometry()`, loop.ts:894: the cell grid the list was built on. */
  cellGeometry(): { readonly divisions: readonly number[]; readonly extent: readonly number[] } {
    return addon.cellGeometry(this.handle);
  }

  /** `StepLoop.passesPerStep`, loop.ts:1105: kernel launches one step makes. */
  get passesPerStep(): number {
    return addon.passesPerStep(this.handle);
  }

  /**
   * `StepLoop.report_pool`, loop.ts:1109: the engine's device allocations.
   * Every allocation is a named one made when the engine is built; there is
   * no scratch pool and nothing is leased.
   */
  report_pool(): PoolReport {
    const m = addon.memory(this.handle);
    return {
      namedCount: m.count,
      namedBytes: m.totalBytes,
      scratchCount: 0,
      scratchBytes: 0,
      totalBytes: m.totalBytes,
      peakBytes: m.totalBytes,
      outstandingLeases: 0,
    };
  }

  destroy(): { leaked: number } {
    return addon.destroy(this.handle);
  }
}
