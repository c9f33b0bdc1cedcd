"""SolidMechanicsModel over the C ABI of libakb.so.

Mirrors the reference's Python binding (python/py_solid_mechanics_model.cc:34-106)
for the explicit path: initFull(_analysis_method=_explicit_lumped_mass),
getStableTimeStep, setTimeStep, solveStep, getEnergy and the nodal-field
getters. The nodal arrays live on the GPU; get*() returns a host mirror that
is refreshed in place on every get*() call, and a mirror handed out by get*()
is written back to the GPU before the next call that uses the state, so
in-place edits of the returned arrays reach the model as in the reference.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _abi
from ._lib import check, lib
from .mesh import element_properties

_explicit_lumped_mass = 0

_FIELD_BY_NAME = {
    "displacement": _abi.FIELD_DISPLACEMENT,
    "velocity": _abi.FIELD_VELOCITY,
    "acceleration": _abi.FIELD_ACCELERATION,
    "external_force": _abi.FIELD_EXTERNAL_FORCE,
    "internal_force": _abi.FIELD_INTERNAL_FORCE,
    "mass": _abi.FIELD_MASS,
}
_WRITABLE = (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY, _abi.FIELD_ACCELERATION,
             _abi.FIELD_EXTERNAL_FORCE)
_ENERGY = {"kinetic": _abi.ENERGY_KINETIC, "potential": _abi.ENERGY_POTENTIAL,
           "external work": _abi.ENERGY_EXTERNAL_WORK}


class Material:
    """Parameters of one `material <law> [ ... ]` section (Material::registerParam
    names: rho, E, nu, Plane_Stress, finite_deformation)."""

    kind = _abi.MATERIAL_ELASTIC

    def __init__(self, rho, E, nu=0.0, Plane_Stress=False, finite_deformation=False,
                 name=""):
        self.name = name
        self.params = dict(rho=float(rho), E=float(E), nu=float(nu),
                           Plane_Stress=bool(Plane_Stress),
                           finite_deformation=bool(finite_deformation))

    def getReal(self, key):
        return self.params[key]

    def getElementFilter(self, el_type, ghost_type=0):
        """Indices of the elements of this material (set by the model's
        initFull; Material::getElementFilter)."""
        if ghost_type != 0:
            raise ValueError("a single GPU holds no ghost elements")
        elements = getattr(self, "_elements", None)
        if elements is None:
            raise RuntimeError("the material belongs to no initialised model")
        return elements

    @property
    def element_filter(self):
        return self.getElementFilter

    def getGradU(self, el_type, ghost_type=0):
        """The displacement gradient at this material's quadrature points
        (Material::getGradU): (points, d*d), rows of column-major matrices
        as the reference's bindings hand them out, the material's elements
        in order; a copy of the model's field at the current displacement."""
        return self._rows(_abi.FIELD_GRAD_U, el_type, ghost_type)

    def getStress(self, el_type, ghost_type=0):
        """The stress at this material's quadrature points (Material::getStress),
        laid out as getGradU."""
        return self._rows(_abi.FIELD_STRESS, el_type, ghost_type)

    def _rows(self, field, el_type, ghost_type):
        ref = getattr(self, "_model", None)
        model = ref() if ref is not None else None  # a weak reference: no cycle
        if model is None:
            raise RuntimeError("the material belongs to no initialised model")
        if el_type != model.mesh.element_type:
            raise ValueError("the material has no elements of type %r" % (el_type,))
        elements = self.getElementFilter(el_type, ghost_type)
        rows = (elements[:, None] * model.nqp + np.arange(model.nqp)[None, :]).reshape(-1)
        return model.getField(field)[rows]

    def desc(self):
        p = self.params
        return _abi.MaterialDesc(self.kind, int(p["Plane_Stress"]),
                                 int(p["finite_deformation"]), 0, p["rho"], p["E"], p["nu"])


class MaterialElastic(Material):
    kind = _abi.MATERIAL_ELASTIC


class MaterialNeohookean(Material):
    kind = _abi.MATERIAL_NEOHOOKEAN

    def __init__(self, rho, E=None, nu=None, lambda_=None, mu=None, **kw):
        if E is None:  # from Lame coefficients
            nu = lambda_ / (2 * (lambda_ + mu))
            E = mu * (3 * lambda_ + 2 * mu) / (lambda_ + mu)
        super().__init__(rho, E, nu, finite_deformation=True, **kw)


class MaterialUser(Material):
    """A material written outside the library: the Material::computeStress
    plugin (material.hh:110; registered through MaterialFactory,
    material.hh:59, 670-691, in the reference). Subclass it and override
    computeStress(grad_u, stress): both are (E*q, d, d) torch CUDA tensors
    viewing the model's device arrays ([k, i, j] = du_i/dX_j at quadrature
    point k); write into stress in place the Cauchy stress (small strain) or
    the first Piola-Kirchhoff stress (finite_deformation=True). rho, E and nu
    give the density and the wave speed of getStableTimeStep."""
    kind = _abi.MATERIAL_USER

    def __init__(self, rho, E, nu=0.0, finite_deformation=True, **kw):
        super().__init__(rho=rho, E=E, nu=nu, finite_deformation=finite_deformation, **kw)

    def computeStress(self, grad_u, stress):
        raise NotImplementedError


def torch_stream(device):
    """cudaStream_t of torch's current stream on a device. torch's default
    stream is the legacy NULL stream, for which the library (where NULL means
    "a stream of its own") is given cudaStreamLegacy."""
    import torch
    return torch.cuda.current_stream(device).cuda_stream or 1


def _device_tensor(ptr, shape, device):
    """Zero-copy torch view of FP64 device memory owned by the library."""
    import torch

    class _Cai:
        __cuda_array_interface__ = dict(shape=tuple(shape), typestr="<f8", data=(int(ptr), False),
                                        version=3, strides=None, stream=None)
    return torch.as_tensor(_Cai(), device="cuda:%d" % device)


def material_from_dict(d):
    kind = d.get("kind", _abi.MATERIAL_ELASTIC)
    cls = MaterialNeohookean if kind == _abi.MATERIAL_NEOHOOKEAN else MaterialElastic
    return cls(rho=d["rho"], E=d["E"], nu=d.get("nu", 0.0),
               **({} if cls is MaterialNeohookean else
                  dict(Plane_Stress=d.get("plane_stress", False),
                       finite_deformation=d.get("finite_deformation", False))))


# axes of the Dirichlet functors (BC::Axis, boundary_condition_functor.hh)
_x, _y, _z = 0, 1, 2


class DirichletFunctor:
    """BC::Dirichlet::DirichletFunctor (boundary_condition_functor.hh,
    py_boundary_conditions.cc): applyBC(functor, group) calls it once per
    node of the group as functor(node, flags, primal, coord) -- flags the
    node's blocked flags (bool, d) and primal its displacement (d), both
    writable; coord its coordinates. Subclass it and define __call__."""

    def __init__(self, axis=_x):
        self.axis = int(axis)

    def __call__(self, node, flags, primal, coord):
        raise NotImplementedError("a DirichletFunctor defines __call__")


class FixedValue(DirichletFunctor):
    """BC::Dirichlet::FixedValue(value, axis)
    (boundary_condition_functor_inline_impl.hh:85-93): the axis blocked, the
    displacement set to value (applied on the device)."""

    def __init__(self, value, axis):
        super().__init__(axis)
        self.value = float(value)

    def __call__(self, node, flags, primal, coord):
        flags[self.axis] = True
        primal[self.axis] = self.value


class IncrementValue(DirichletFunctor):
    """BC::Dirichlet::IncrementValue(value, axis): the axis blocked, value
    added to its displacement."""

    def __init__(self, value, axis):
        super().__init__(axis)
        self.value = float(value)

    def __call__(self, node, flags, primal, coord):
        flags[self.axis] = True
        primal[self.axis] += self.value


class Increment(DirichletFunctor):
    """BC::Dirichlet::Increment(vector): every axis blocked, the vector
    added to the displacement."""

    def __init__(self, increment):
        super().__init__(_x)
        self.increment = np.asarray(increment, dtype=np.float64).reshape(-1)

    def __call__(self, node, flags, primal, coord):
        flags[:] = True
        primal += self.increment


class NeumannFunctor:
    """BC::Neumann::NeumannFunctor (boundary_condition_functor.hh,
    py_boundary_conditions.cc): applyBC(functor, group) calls it at every
    Gauss point of the group's facets as functor(quad_point, dual, coord,
    normals) -- dual (d) to receive the traction there, coord the point's
    coordinates, normals the facet's unit normal -- and adds the integrated
    nodal forces to the external force. Subclass it and define __call__."""

    def __call__(self, quad_point, dual, coord, normals):
        raise NotImplementedError("a NeumannFunctor defines __call__")


class FromTraction(NeumannFunctor):
    """BC::Neumann::FromSameDim (FromTraction in the reference's Python
    package): a traction vector on the group's facets (integrated in the
    library, akb_neumann_forces)."""
    kind = _abi.NEUMANN_TRACTION

    def __init__(self, traction):
        self.traction = np.asarray(traction, dtype=np.float64).reshape(-1)

    def __call__(self, quad_point, dual, coord, normals):
        dual[:] = self.traction

    def akb_value(self, dim):
        if self.traction.size != dim:
            raise ValueError("a traction of %d components in %dD" % (self.traction.size, dim))
        return self.traction


class FromStress(NeumannFunctor):
    """BC::Neumann::FromHigherDim (FromStress in the reference's Python
    package): a stress tensor, the traction sigma n with n each facet's unit
    normal as its node order gives it."""
    kind = _abi.NEUMANN_STRESS

    def __init__(self, stress):
        self.stress = np.asarray(stress, dtype=np.float64)

    def __call__(self, quad_point, dual, coord, normals):
        dual[:] = self.stress @ normals

    def akb_value(self, dim):
        if self.stress.shape != (dim, dim):
            raise ValueError("a %s stress in %dD" % (self.stress.shape, dim))
        return self.stress.T.reshape(-1)  # column-major


class FreeBoundary(NeumannFunctor):
    """BC::Neumann::FreeBoundary: a zero traction (adds nothing)."""

    def __call__(self, quad_point, dual, coord, normals):
        dual[:] = 0.0


FromSameDim = FromTraction
FromHigherDim = FromStress


class SolidMechanicsModel:
    """The explicit lumped-mass SolidMechanicsModel on one GPU."""

    def __init__(self, mesh, materials=None, element_material=None,
                 precision=None, device=0, stream=None,
                 patch_elements=0, patch_nodes=0, interface_nodes=None, patch_grid=0):
        """materials: the model's materials; none given, initFull takes them
        from the sections of the last parseInput (the reference's
        SolidMechanicsModel(mesh)), laws written in Python included
        (akantu_b200.material_plugin). element_material: the material of
        each element (default: the first material, the reference's default
        selector). precision: AKB_MODE_*; default AKB_MODE_FP64_REFERENCE,
        or AKB_MODE_FP64 for laws written in Python (their only mode).
        interface_nodes: this model is one part of a partitioned mesh
        (akb_model_create_part), these of its nodes are shared with other
        parts; step it through akantu_b200.decompose.DistributedModel.
        patch_elements, patch_nodes, patch_grid: the fused step's patch shape
        and schedule (akb_model_options; 0 = defaults)."""
        self.mesh = mesh
        self._iface = None if interface_nodes is None else \
            np.ascontiguousarray(interface_nodes, dtype=np.uint32)
        self.dim, self.nnpe, self.nqp = element_properties(mesh.element_type)
        self._materials = list(materials) if materials else []
        self._element_material = element_material
        self._precision = precision
        self._device = device
        self._stream = stream
        self._patch = (int(patch_elements), int(patch_nodes), int(patch_grid))
        self._h = None
        self._user = []
        self._mirrors = {}
        self._views = {}
        self._checked_out = set()
        self._blocked = None
        self._laws = None  # material_plugin.LawBridge of laws written in Python
        self._qp_weights = None
        self._selector = None

    # -- initialisation --------------------------------------------------
    def addMaterial(self, material):
        self._materials.append(material)

    def setMaterialSelector(self, selector):
        """setMaterialSelector (solid_mechanics_model.hh): the element ->
        material map initFull takes, e.g. a
        material_plugin.MeshDataMaterialSelectorString."""
        self._selector = selector

    def initFull(self, _analysis_method=_explicit_lumped_mass, precision=None):
        if _analysis_method != _explicit_lumped_mass:
            raise NotImplementedError("only _explicit_lumped_mass is on this path")
        if precision is not None:
            self._precision = precision
        if not self._materials:
            self._materials_from_input()
        elif self._selector is not None and self._element_material is None:
            self._element_material = self._selector.select([m.name for m in self._materials])
        if self._precision is None:
            self._precision = _abi.MODE_FP64_REFERENCE
        em = (np.zeros(self.mesh.getNbElement(), dtype=np.int64) if self._element_material is None
              else np.asarray(self._element_material, dtype=np.int64))
        for k, m in enumerate(self._materials):
            m._elements = np.nonzero(em == k)[0]
            m._model = weakref.ref(self)
        L = lib()
        self._nodes = np.ascontiguousarray(self.mesh.nodes, dtype=np.float64)
        self._conn = np.ascontiguousarray(self.mesh.connectivity, dtype=np.uint32)
        desc = _abi.MeshDesc(self.dim, self.mesh.element_type, self._nodes.shape[0],
                             self._conn.shape[0],
                             self._nodes.ctypes.data_as(C.POINTER(C.c_double)),
                             self._conn.ctypes.data_as(C.POINTER(C.c_uint32)))
        mats = (_abi.MaterialDesc * len(self._materials))(*[m.desc() for m in self._materials])
        em = None
        if self._element_material is not None:
            self._em = np.ascontiguousarray(self._element_material, dtype=np.uint32)
            em = self._em.ctypes.data_as(C.POINTER(C.c_uint32))
        self._user = [m for m in self._materials if isinstance(m, MaterialUser)]
        if self._user and self._stream is None:
            # user stresses are computed with torch: share its stream
            self._stream = torch_stream(self._device)
        opt = _abi.ModelOptions(self._precision, self._device, self._stream, *self._patch)
        h = C.c_void_p()
        if self._iface is None:
            check(L.akb_model_create(C.byref(desc), len(self._materials), mats, em,
                                     C.byref(opt), C.byref(h)))
        else:
            check(L.akb_model_create_part(C.byref(desc), len(self._materials), mats, em,
                                          C.byref(opt),
                                          self._iface.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          self._iface.size, C.byref(h)))
        self._h = h

    def _materials_from_input(self):
        """The materials of the last parseInput's sections: the laws the
        library computes become device materials, the others are allocated
        by MaterialFactory and run in Python (material_plugin.LawBridge)."""
        from . import material_plugin as mp
        sections = mp.input_sections()
        if not sections:
            raise ValueError("no material: pass materials, addMaterial() or parseInput() first")
        if self._element_material is None:
            if self._selector is not None:
                names = [str(prm.get("name", "%s_%d" % (law, k)))
                         for k, (law, prm) in enumerate(sections)]
                self._element_material = self._selector.select(names)
            else:  # the default selector: every element takes the first material
                self._element_material = np.zeros(self.mesh.getNbElement(), dtype=np.uint32)
        builtin = [law in mp.BUILTIN_LAWS for law, _ in sections]
        if all(builtin):
            for law, prm in sections:
                cls = MaterialNeohookean if law == "neohookean" else MaterialElastic
                kw = {} if cls is MaterialNeohookean else dict(
                    Plane_Stress=bool(prm.get("Plane_Stress", False)),
                    finite_deformation=bool(prm.get("finite_deformation", False)))
                self._materials.append(cls(rho=prm.get("rho", 0.0), E=prm.get("E", 0.0),
                                           nu=prm.get("nu", 0.5),  # the reference's default
                                           name=str(prm.get("name", law)), **kw))
            return
        if any(builtin):
            raise ValueError("laws written in Python and built-in laws in one model: the "
                             "library steps a model with either kind, not both")
        laws = [mp.law_from_section(law, prm, k, self.dim, self)
                for k, (law, prm) in enumerate(sections)]
        self._laws = mp.LawBridge(laws, self._element_material, self.mesh.element_type,
                                  self.nqp, self.dim)
        for law in laws:
            law.initMaterial()
            # the library's wave speed sqrt((lambda + 2 mu) / rho) with nu = 0
            # is sqrt(E / rho): E = rho c^2 carries the law's push wave speed
            c = float(law.getPushWaveSpeed(None))
            rho = law.getReal("rho")
            self._materials.append(MaterialUser(rho=rho, E=rho * c * c, nu=0.0,
                                                finite_deformation=law.finite_deformation,
                                                name=law.name))
        if self._precision is None:
            self._precision = _abi.MODE_FP64

    def getMaterialIndex(self, name):
        laws = self._laws.laws if self._laws is not None else self._materials
        for k, m in enumerate(laws):
            if m.name == name:
                return k
        raise KeyError("no material named %r" % name)

    def getMaterial(self, key):
        """The material with this index or name (a law written in Python: its
        Material object)."""
        laws = self._laws.laws if self._laws is not None else self._materials
        if isinstance(key, str):
            for m in laws:
                if m.name == key:
                    return m
            raise KeyError("no material named %r" % key)
        return laws[key]

    def __del__(self):
        self.close()

    def close(self):
        self._views = {}  # views of the device arrays about to be freed
        if getattr(self, "_h", None):
            lib().akb_model_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("call initFull() first")
        return self._h

    def getInfo(self):
        info = _abi.ModelInfo()
        check(lib().akb_model_get_info(self.handle, C.byref(info)))
        return info

    # -- host mirrors ------------------------------------------------------
    def _sync_in(self):
        for f in list(self._checked_out):
            arr = self._mirrors[f]
            check(lib().akb_set_field(self.handle, f, arr.ctypes.data_as(C.POINTER(C.c_double)),
                                      arr.size))
        self._checked_out.clear()
        if self._blocked is not None:
            b = self._blocked
            check(lib().akb_set_blocked_dofs(self.handle, b.ctypes.data_as(C.POINTER(C.c_uint8)),
                                             b.size))
            self._blocked = None

    def getField(self, field):
        self._sync_in()
        n = self.mesh.getNbNodes() * self.dim
        if field in (_abi.FIELD_GRAD_U, _abi.FIELD_STRESS):
            n = self.mesh.getNbElement() * self.nqp * self.dim * self.dim
        arr = self._mirrors.get(field)
        if arr is None or arr.size != n:
            cols = self.dim * self.dim if field in (_abi.FIELD_GRAD_U, _abi.FIELD_STRESS) else self.dim
            arr = np.zeros((n // cols, cols))
            self._mirrors[field] = arr
        check(lib().akb_get_field(self.handle, field, arr.ctypes.data_as(C.POINTER(C.c_double)), n))
        if field in _WRITABLE:
            self._checked_out.add(field)
        return arr

    def setField(self, field, values):
        self._sync_in()
        arr = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        check(lib().akb_set_field(self.handle, field, arr.ctypes.data_as(C.POINTER(C.c_double)),
                                  arr.size))
        if field in self._mirrors:
            self._mirrors[field][...] = arr.reshape(self._mirrors[field].shape)

    def getDisplacement(self):
        return self.getField(_abi.FIELD_DISPLACEMENT)

    def getVelocity(self):
        return self.getField(_abi.FIELD_VELOCITY)

    def getAcceleration(self):
        return self.getField(_abi.FIELD_ACCELERATION)

    def getExternalForce(self):
        return self.getField(_abi.FIELD_EXTERNAL_FORCE)

    def getInternalForce(self):
        return self.getField(_abi.FIELD_INTERNAL_FORCE)

    def getMass(self):
        return self.getField(_abi.FIELD_MASS)

    def getBlockedDOFs(self):
        """Host array of blocked flags (bool, N x d); edits are applied before
        the next solveStep()."""
        self._sync_in()
        b = np.zeros((self.mesh.getNbNodes(), self.dim), dtype=np.uint8)
        check(lib().akb_get_blocked_dofs(self.handle, b.ctypes.data_as(C.POINTER(C.c_uint8)),
                                         b.size))
        view = b.view(np.bool_)
        self._blocked = b
        return view

    def setBlockedDOFs(self, blocked):
        self._sync_in()
        b = np.ascontiguousarray(blocked, dtype=np.uint8).reshape(-1)
        check(lib().akb_set_blocked_dofs(self.handle, b.ctypes.data_as(C.POINTER(C.c_uint8)),
                                         b.size))

    def applyDirichlet(self, nodes, component, values):
        """applyBC(FixedValue(value, axis), group) for a node group
        (boundary_condition_tmpl.hh:63-200): blocks the DOFs and sets their
        displacement on the device. component _abi.ALL_COMPONENTS: every axis
        at once, values (nb_nodes, dim)."""
        self._sync_in()
        n = np.ascontiguousarray(nodes, dtype=np.uint32)
        shape = n.shape + ((self.dim,) if component == _abi.ALL_COMPONENTS else ())
        v = np.ascontiguousarray(np.broadcast_to(values, shape), dtype=np.float64)
        check(lib().akb_apply_dirichlet(self.handle, n.ctypes.data_as(C.POINTER(C.c_uint32)),
                                        n.size, int(component),
                                        v.ctypes.data_as(C.POINTER(C.c_double))))

    def applyBC(self, functor, group):
        """applyBC(functor, group) (py_solid_mechanics_model.cc:58-67,
        boundary_condition_tmpl.hh) on a mesh group (a `$PhysicalNames`
        group, or one created with Mesh.createNodeGroup; a Dirichlet functor
        also takes a node list). A Dirichlet functor acts on the group's
        nodes: FixedValue on the device, any other (IncrementValue, Increment,
        a DirichletFunctor written in Python) node by node on the host. A
        Neumann functor adds the nodal forces of its traction on the group's
        facets to the external force: FromTraction / FromStress integrated in
        the library, a NeumannFunctor written in Python at the facets' Gauss
        points (boundary_condition_tmpl.hh:95-185)."""
        if isinstance(functor, NeumannFunctor):
            if not isinstance(group, str):
                raise TypeError("a Neumann condition acts on a named group's facets")
            forces = self.mesh.neumannForces(group, functor)
            f = self.getExternalForce()  # ADDED, as the reference assembles it
            f += forces
            return
        if not isinstance(functor, DirichletFunctor):
            raise TypeError("applyBC takes a DirichletFunctor or a NeumannFunctor")
        nodes = self.mesh.getNodeGroup(group) if isinstance(group, str) else np.asarray(group)
        if type(functor) is FixedValue:
            self.applyDirichlet(nodes, functor.axis, functor.value)
            return
        u = np.array(self.getField(_abi.FIELD_DISPLACEMENT))
        b = self.getBlockedDOFs().copy()
        X = np.asarray(self.mesh.nodes, dtype=np.float64)
        for node in np.asarray(nodes, dtype=np.int64):
            functor(int(node), b[node], u[node], X[node])
        self.setField(_abi.FIELD_DISPLACEMENT, u)
        self.setBlockedDOFs(b)

    def getGradU(self):
        return self.getField(_abi.FIELD_GRAD_U)

    def getStress(self):
        return self.getField(_abi.FIELD_STRESS)

    # -- solver --------------------------------------------------------------
    def assembleMassLumped(self):
        check(lib().akb_assemble_mass_lumped(self.handle))

    def getStableTimeStep(self):
        self._sync_in()
        dt = C.c_double()
        check(lib().akb_get_stable_time_step(self.handle, C.byref(dt)))
        return dt.value

    def setTimeStep(self, time_step, solver_id=""):
        check(lib().akb_set_time_step(self.handle, float(time_step)))

    def getTimeStep(self):
        dt = C.c_double()
        check(lib().akb_get_time_step(self.handle, C.byref(dt)))
        return dt.value

    def solveStep(self, solver_id=""):
        self._sync_in()
        if self._user:
            self.stepBegin()
            G, S = self.deviceTensor(_abi.FIELD_GRAD_U), self.deviceTensor(_abi.FIELD_STRESS)
            if self._laws is not None:
                self._laws.stresses(G, S)
            else:
                self._user[0].computeStress(G, S)
            self.stepEnd()
            return
        check(lib().akb_solve_step(self.handle))

    def solveSteps(self, nb_steps):
        """nb_steps solveStep() calls replayed from a CUDA graph."""
        self._sync_in()
        if self._user:
            for _ in range(int(nb_steps)):
                self.solveStep()
            return
        check(lib().akb_solve_steps(self.handle, int(nb_steps)))

    def stepBegin(self):
        """Predictor and grad u at the quadrature points (user materials)."""
        self._sync_in()
        check(lib().akb_step_begin(self.handle))

    def stepEnd(self):
        """Internal forces from the stress field, lumped solve, corrector."""
        check(lib().akb_step_end(self.handle))

    def stream(self):
        p = C.c_void_p()
        check(lib().akb_model_get_stream(self.handle, C.byref(p)))
        return p.value

    def deviceTensor(self, field):
        """Zero-copy torch view of a device field: (N, d) nodal fields, or
        (E*q, d, d) [k, i, j] quadrature fields (column-major storage). The
        views are cached per field while the field's device address stays
        the same (a user material's step asks for two every step)."""
        ptr = self.devicePointer(field)
        cached = self._views.get(field)
        if cached is not None and cached[0] == ptr:
            return cached[1]
        if field in (_abi.FIELD_GRAD_U, _abi.FIELD_STRESS):
            n = self.mesh.getNbElement() * self.nqp
            t = _device_tensor(ptr, (n, self.dim, self.dim), self._device).transpose(1, 2)
        else:
            t = _device_tensor(ptr, (self.mesh.getNbNodes(), self.dim), self._device)
        self._views[field] = (ptr, t)
        return t

    def timeSolveSteps(self, nb_steps):
        """Device time (ms) of nb_steps steps, CUDA events on the model's stream."""
        self._sync_in()
        ms = C.c_double()
        check(lib().akb_time_solve_steps(self.handle, int(nb_steps), C.byref(ms)))
        return ms.value

    def assembleInternalForces(self):
        self._sync_in()
        check(lib().akb_assemble_internal_forces(self.handle))

    def computeStresses(self):
        self._sync_in()
        check(lib().akb_compute_stresses(self.handle))

    def getEnergy(self, energy_id):
        self._sync_in()
        if self._laws is not None and energy_id == "potential":
            from .material_plugin import qp_weights
            if self._qp_weights is None:
                self._qp_weights = qp_weights(self.mesh)
            return self._laws.potential_energy(self._qp_weights)
        v = C.c_double()
        check(lib().akb_get_energy(self.handle, _ENERGY[energy_id], C.byref(v)))
        return v.value

    def getEnergyAsync(self, energy_id, out):
        """getEnergy queued on the model's stream: the value lands in out (a
        pinned host or device float64 buffer of one element, as a pointer or
        a tensor/array) when the stream reaches it; read it after
        synchronize()."""
        self._sync_in()
        ptr = out if isinstance(out, int) else (out.data_ptr() if hasattr(out, "data_ptr")
                                                else out.ctypes.data)
        check(lib().akb_get_energy_async(self.handle, _ENERGY[energy_id], C.c_void_p(ptr)))

    def synchronize(self):
        check(lib().akb_synchronize(self.handle))

    def devicePointer(self, field):
        p = C.c_void_p()
        check(lib().akb_field_device_pointer(self.handle, field, C.byref(p)))
        return p.value
