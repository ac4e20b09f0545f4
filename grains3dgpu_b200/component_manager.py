"""Python mirror of Grains3D's ComponentManager hot path over the C ABI.

Method names and call order follow ComponentManager<T>
(Grains/Component/include/ComponentManager.hh:37-182) and the time loop of
GrainsCPU::simulate (Grains/Base/src/GrainsCPU.cpp:46-70), so a driver written
against the reference reads the same:

    cm = ComponentManagerB200(scene)
    for t in times:
        cm.detectCollisionAndComputeContactForces(result)
        cm.addExternalForces()
        cm.moveParticles()

Transforms are (N, 12) arrays (basis row-major + origin, Transform3's
buffer), velocities (N, 6) (translational + angular, Kinematics), torces
(N, 6) (force + torque).  Errors raise :class:`EngineError` with the engine's
status; an out-of-domain particle is reported through ``last_status``.
"""
import numpy as np

from . import abi, engine, scenes


class EngineError(RuntimeError):
    def __init__(self, what, status):
        super().__init__(f"{what}: {engine.status_string(status)} ({status})")
        self.status = status


class ComponentManagerB200:
    def __init__(self, scene, **config_overrides):
        self._lib = engine.load()
        self.scene = scene
        try:
            self._sys = scenes.System(self._lib, scene, **config_overrides)
        except RuntimeError as e:
            raise EngineError(str(e), abi.GB_E_INVALID_ARG) from e
        self.last_status = abi.GB_OK

    # ---- ComponentManager getters/setters ----------------------------------------
    def getNumberOfParticles(self):
        return self._sys.n

    def getNumberOfObstacles(self):
        return self._sys.cfg.n_obstacles

    def getNumberOfCells(self):
        return self._sys.stats().n_cells

    def getRigidBodyId(self):
        return self.scene.rb_ids.copy()

    def getTransform(self):
        return self._sys.transforms()

    def setTransform(self, tr):
        self._sys.set_transforms(np.asarray(tr, np.float64).reshape(-1, 12))

    def getVelocity(self):
        return self._sys.velocities()

    def setVelocity(self, kin):
        self._sys.set_velocities(np.asarray(kin, np.float64).reshape(-1, 6))

    def getTorce(self):
        return self._sys.torces()

    # ---- the hot path ---------------------------------------------------------------
    def _call(self, what, st):
        self.last_status = st
        if st not in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN):
            raise EngineError(what, st)
        return st

    def updateLinks(self):
        return self._call("updateLinks", self._lib.update_links(self._sys.ctx))

    def detectCollisionAndComputeContactForces(self, result=None):
        if result is not None:
            assert result.dtype == np.int32 and result.shape == (self._sys.n,)
        return self._call("detectCollisionAndComputeContactForces",
                          self._lib.detect_collision_and_compute_contact_forces(
                              self._sys.ctx, abi.i32ptr(result)))

    def addExternalForces(self):
        return self._call("addExternalForces", self._lib.add_external_forces(self._sys.ctx))

    def moveParticles(self):
        return self._call("moveParticles", self._lib.move_particles(self._sys.ctx))

    def step(self, n=1):
        """n iterations of GrainsCPU::simulate's loop body, fused on the device."""
        return self._call("step", self._lib.step(self._sys.ctx, n))

    def stats(self):
        return self._sys.stats()

    def dump(self, kind):
        return self._sys.dump(kind)

    def close(self):
        self._sys.close()
