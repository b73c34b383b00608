"""Host-side driver over the libe4cuda C ABI.

``Simulation`` plays the part of the D host's ``simcore`` for this path
(src/eilmer/simcore.d): it owns the configuration, creates the blocks
(``init_simulation`` :180), uploads the initial flow state (:305-322) and
advances the solution with ``integrate_in_time`` (:791).  Every step runs on
the GPU through the C ABI; nothing here computes flow physics.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .config import make_config


@dataclass
class RunInfo:
    steps_taken: int
    time: float
    dt_global: float
    status: int
    status_step: int
    bad_cells: int


class Simulation:
    """One set of structured blocks sharing dt_global, resident on one GPU."""

    def __init__(self, config: dict | None = None, control: dict | None = None, *,
                 precision: str = "fp64", device: int = 0, use_graphs: bool = True,
                 gas: dict | None = None, thermochem=None):
        self.L = _lib.load()
        if thermochem is not None:
            gas = dict(gas or {}, model="therm_perf_5sp_air")
        self.cfg = make_config(config, control, precision=precision, device=device,
                               use_graphs=use_graphs, gas=gas)
        _lib.check(self.L.e4c_init(self.cfg))
        self.blocks = []   # (ni, nj, nk)
        self.vertices = []
        self.species = ["air"]
        self.nsp = 1
        if thermochem is not None:
            self._tc = thermochem.fill(_lib.E4CThermoChem())
            _lib.check(self.L.e4c_set_thermochem(ctypes.byref(self._tc)))
            self.nsp = thermochem.nsp
            self.species = list(thermochem.species)

    @classmethod
    def from_workload(cls, wl, *, precision="fp64", control=None, use_graphs=True, **config):
        device = int(config.pop("device", 0))
        cfgd = {"dimensions": wl.dimensions, "flux_calculator": wl.flux_calculator}
        cfgd.update(config)
        tc = getattr(wl, "thermochem", None)
        sim = cls(cfgd, control, precision=precision, device=device, use_graphs=use_graphs,
                  thermochem=tc)
        for b in wl.blocks:
            h = sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
            sim.upload(h, b.prim)
        return sim

    def close(self):
        if getattr(self, "L", None) is not None:
            self.L.e4c_finalize()
            self.L = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_block(self, ni, nj, nk, vtx, bc, inflow) -> int:
        vtx = np.ascontiguousarray(vtx, dtype=np.float64)
        inflow = np.ascontiguousarray(inflow, dtype=np.float64)
        bca = (ctypes.c_int * 6)(*bc)
        h = _lib.check(self.L.e4c_block_create(ni, nj, nk, _lib.dptr(vtx), bca, _lib.dptr(inflow)))
        nk_eff = nk if self.cfg.dimensions == 3 else 1
        self.blocks.append((ni, nj, nk_eff))
        self.vertices.append(vtx)
        return h

    def connect(self, ha, face_a, hb, face_b, orientation=0):
        """Join face face_a of block ha to face face_b of block hb with an
        exchange boundary (any face pair, orientation 0..3 in 3-D)."""
        _lib.check(self.L.e4c_connect_blocks(int(ha), int(face_a), int(hb), int(face_b),
                                             int(orientation)))

    def ncell(self, h):
        ni, nj, nk = self.blocks[h]
        return ni * nj * nk

    def upload(self, h, prim):
        """prim: (8, ncell) float64 numpy array or a contiguous (pinned) torch tensor."""
        if not hasattr(prim, "data_ptr"):
            prim = np.ascontiguousarray(prim, dtype=np.float64)
            assert prim.shape[-1] == self.ncell(h)
        _lib.check(self.L.e4c_block_upload(h, _lib.dptr(prim)))

    def upload_cons(self, h, cons):
        """cons: (5, ncell) conserved state (ideal gas), decoded on the device as
        the end of a stage decodes it, so a run continues bit for bit."""
        if not hasattr(cons, "data_ptr"):
            cons = np.ascontiguousarray(cons, dtype=np.float64)
            assert cons.shape == (5, self.ncell(h))
        _lib.check(self.L.e4c_block_upload_cons(h, _lib.dptr(cons)))

    def download(self, h, prim=None, cons=None, want_cons=True):
        """Primitive (8, ncell) and conserved (5, ncell) state; the outputs may be
        given (numpy arrays or contiguous pinned torch tensors)."""
        n = self.ncell(h)
        ns = self.nsp if self.nsp > 1 else 0
        if prim is None:
            prim = np.zeros((8 + ns, n))
        if cons is None and want_cons:
            cons = np.zeros((5 + ns, n))
        _lib.check(self.L.e4c_block_download(h, _lib.dptr(prim),
                                             _lib.dptr(cons) if cons is not None else None))
        return prim, cons

    def upload_async(self, h, prim):
        """Queue an upload from a contiguous pinned host tensor/array (returns
        at once; call wait_transfers before reusing the host buffer)."""
        _lib.check(self.L.e4c_block_upload_async(h, _lib.dptr(prim)))

    def upload_cons_async(self, h, cons):
        """Queue a conserved-state upload (see upload_cons) from a contiguous
        pinned host tensor/array."""
        _lib.check(self.L.e4c_block_upload_cons_async(h, _lib.dptr(cons)))

    def download_async(self, h, prim=None, cons=None):
        """Queue a download into contiguous pinned host buffers."""
        _lib.check(self.L.e4c_block_download_async(
            h, _lib.dptr(prim) if prim is not None else None,
            _lib.dptr(cons) if cons is not None else None))

    def run_async(self, nsteps, max_time=1.0e300):
        """Queue nsteps steps without waiting (status: next run())."""
        _lib.check(self.L.e4c_integrate_async(int(nsteps), float(max_time)))

    def wait_transfers(self):
        _lib.check(self.L.e4c_transfers_wait())

    def run(self, nsteps, max_time=1.0e300) -> RunInfo:
        info = _lib.E4CRunInfo()
        rc = self.L.e4c_integrate(int(nsteps), float(max_time), ctypes.byref(info))
        _lib.check(rc)
        return RunInfo(info.steps_taken, info.time, info.dt_global, info.status,
                       info.status_step, info.bad_cells)

    def dt_allow(self, hs, dt_current, check_cfl):
        arr = (ctypes.c_int * len(hs))(*hs)
        d, c = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.e4c_dt_allow(arr, len(hs), float(dt_current), int(bool(check_cfl)),
                                       ctypes.byref(d), ctypes.byref(c)))
        return d.value, c.value

    def gasdynamic_step(self, hs, dt):
        arr = (ctypes.c_int * len(hs))(*hs)
        bad = ctypes.c_int()
        _lib.check(self.L.e4c_gasdynamic_step(arr, len(hs), float(dt), ctypes.byref(bad)))
        return bad.value

    def stage(self, hs, stage, dt):
        """One stage of the gas-dynamic step (the last one ends the step);
        returns the stage's invalid-cell count."""
        arr = (ctypes.c_int * len(hs))(*hs)
        bad = ctypes.c_int()
        _lib.check(self.L.e4c_stage(arr, len(hs), int(stage), float(dt), ctypes.byref(bad)))
        return bad.value

    # -- faces joined to blocks on other ranks (sharding.py) -----------------
    def connect_remote(self, h, face):
        _lib.check(self.L.e4c_connect_remote(int(h), int(face)))

    def face_slab_bytes(self, h, face):
        n = ctypes.c_longlong()
        _lib.check(self.L.e4c_face_slab_bytes(int(h), int(face), ctypes.byref(n)))
        return n.value

    def pack_face(self, h, face, stage, dev_ptr):
        _lib.check(self.L.e4c_pack_face(int(h), int(face), int(stage), ctypes.c_void_p(dev_ptr)))

    def unpack_face(self, h, face, dev_ptr):
        _lib.check(self.L.e4c_unpack_face(int(h), int(face), ctypes.c_void_p(dev_ptr)))

    def chemistry_step(self, hs, dt):
        arr = (ctypes.c_int * len(hs))(*hs)
        _lib.check(self.L.e4c_chemistry_step(arr, len(hs), float(dt)))

    def chemistry_counters(self, reset=False):
        """(reacting cells, Newton iterations, recovered cells, Newton-active
        cells) accumulated by the chemistry updates since the last reset."""
        out = (ctypes.c_longlong * 4)()
        _lib.check(self.L.e4c_chemistry_counters(out, int(bool(reset))))
        return tuple(int(x) for x in out)

    # -- flow files (sfluidblock.d:1778-1956) --------------------------------
    def write_flow(self, h, path, fmt="gziptext", label=""):
        """Write block h's current state as an Eilmer4 flow file."""
        from . import flowfile
        ni, nj, nk = self.blocks[h]
        dims = self.cfg.dimensions
        prim, _ = self.download(h, want_cons=False)
        pos, vol = flowfile.cell_geometry(self.vertices[h], ni, nj, nk, dims)
        dt_chem = None
        if self.nsp > 1 and self.cfg.reacting:
            dt_chem = np.zeros(ni * nj * nk)
            _lib.check(self.L.e4c_block_get_dt_chem(h, _lib.dptr(dt_chem)))
        t, _, _ = self.state()
        flowfile.write_flow(path, prim=prim, pos=pos, volume=vol, dimensions=dims, ni=ni, nj=nj,
                            nk=nk, species=self.species, sim_time=t, label=label,
                            dt_chem=dt_chem, fmt=fmt)

    def read_flow(self, h, path, fmt="gziptext"):
        """Set block h's state from an Eilmer4 flow file; returns its sim_time."""
        from . import flowfile
        fl = flowfile.read_flow(path, fmt)
        if (fl["nicell"], fl["njcell"], fl["nkcell"]) != self.blocks[h]:
            raise ValueError("the flow file's block size differs from block %d" % h)
        prim, dt_chem = flowfile.prim_from_flow(fl, self.nsp)
        self.upload(h, prim)
        if dt_chem is not None and self.cfg.reacting:
            dt_chem = np.ascontiguousarray(dt_chem)
            _lib.check(self.L.e4c_block_set_dt_chem(h, _lib.dptr(dt_chem)))
        return fl["sim_time"]

    # -- learned chemistry seed ---------------------------------------------
    def seed_collect(self, hs, dt, nsamples, seed=1):
        """Add nsamples (state, dt) -> plain-update pairs from the blocks' hot cells."""
        arr = (ctypes.c_int * len(hs))(*hs)
        _lib.check(self.L.e4c_seed_collect(arr, len(hs), float(dt), int(nsamples), int(seed)))

    def seed_dataset(self):
        n = ctypes.c_longlong()
        _lib.check(self.L.e4c_seed_dataset(ctypes.byref(n)))
        return n.value

    def seed_clear(self):
        _lib.check(self.L.e4c_seed_clear())

    def seed_train(self, epochs=8, batch=2048, lr=2.0e-3, seed=1):
        """Train on the collected pairs; returns the training report."""
        rep = (ctypes.c_double * 6)()
        _lib.check(self.L.e4c_seed_train(int(epochs), int(batch), float(lr), int(seed), rep))
        keys = ("train_loss", "val_loss", "n_train", "n_val", "seconds", "steps")
        return dict(zip(keys, list(rep)))

    def seed_get(self):
        p = np.zeros(_lib.SEED_NPARAM, dtype=np.float32)
        norm = np.zeros(_lib.SEED_NNORM)
        _lib.check(self.L.e4c_seed_get(_lib.fptr(p), _lib.dptr(norm)))
        return p, norm

    def seed_set(self, params, norm):
        p = np.ascontiguousarray(params, dtype=np.float32)
        nm = np.ascontiguousarray(norm, dtype=np.float64)
        assert p.size == _lib.SEED_NPARAM and nm.size == _lib.SEED_NNORM
        _lib.check(self.L.e4c_seed_set(_lib.fptr(p), _lib.dptr(nm)))

    def seed_enable(self, on=True):
        _lib.check(self.L.e4c_seed_enable(int(bool(on))))

    def seed_predict(self, rows):
        """rows (n, 8): T, p, Y[5], dt -> (n, 6): predicted dY[5], dT."""
        r = np.ascontiguousarray(rows, dtype=np.float64)
        out = np.zeros((r.shape[0], 6))
        _lib.check(self.L.e4c_seed_predict(_lib.dptr(r), r.shape[0], _lib.dptr(out)))
        return out

    def seed_loss_grad(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(_lib.SEED_NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        _lib.check(self.L.e4c_seed_loss_grad(_lib.fptr(x), _lib.fptr(y), x.shape[0],
                                             ctypes.byref(loss), _lib.fptr(g)))
        return loss.value, g

    def state(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _lib.check(self.L.e4c_sim_state(ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)))
        return t.value, dt.value, st.value

    def synchronize(self):
        _lib.check(self.L.e4c_synchronize())

    # -- timing hooks -------------------------------------------------------
    def stream_handle(self) -> int:
        """The cudaStream_t the library enqueues on (as an integer)."""
        return int(self.L.e4c_stream() or 0)

    def kernel_launches(self) -> int:
        return int(self.L.e4c_kernel_launches())

    def profile(self, nsteps):
        """Per kernel class: (total ms, launches) over nsteps graph-free steps."""
        ms = (ctypes.c_double * len(_lib.KCLASS))()
        nl = (ctypes.c_int * len(_lib.KCLASS))()
        _lib.check(self.L.e4c_profile_steps(int(nsteps), ms, nl))
        return {name: (ms[q], nl[q]) for q, name in enumerate(_lib.KCLASS)}

    # -- fused-kernel tile shape -------------------------------------------
    def set_tile(self, ti, tj, kc):
        _lib.check(self.L.e4c_set_tile(int(ti), int(tj), int(kc)))

    def set_flux_runs(self, i_faces, jk_faces):
        """Faces per thread of the row-walking flux kernel (curvilinear 3-D
        ideal-gas blocks); (0, 0) restores the per-block choice."""
        _lib.check(self.L.e4c_set_flux_runs(int(i_faces), int(jk_faces)))

    def get_tile(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self.L.e4c_get_tile(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def autotune(self, nsteps=3):
        """Pick the fastest fused tile shape on the current blocks; the flow
        state and clock are left exactly as they were."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        _lib.check(self.L.e4c_autotune(int(nsteps), ctypes.byref(a), ctypes.byref(b),
                                       ctypes.byref(c), ctypes.byref(ms)))
        return (a.value, b.value, c.value), ms.value
