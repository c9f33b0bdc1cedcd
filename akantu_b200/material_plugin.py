"""Materials written in Python in the reference's plugin style
(python/py_material.cc, python/py_parser.cc): a subclass of Material that
registers its parameters (registerParamReal), reads them (getReal), and
computes the stress of its elements' quadrature points in
computeStress(el_type, ghost_type) from the numpy arrays getGradU and
getStress; registered with MaterialFactory.registerAllocator and
instantiated from the `material <law> [ ... ]` sections of an input file read
by parseInput.

Such a law runs on the host, on copies of its quadrature points' fields made
every step (the reference, too, runs a Python law on host arrays); the
displacement gradient, the internal forces and the central-difference update
stay on the GPU (akb_step_begin / akb_step_end). A section whose law the
library implements (elastic, neohookean) becomes a device material instead;
one model holds either kind, not both (akb_model_create).

Array layout, as the reference's bindings hand it out: getGradU(el_type) and
getStress(el_type) are (points, d*d) arrays whose rows are column-major
d x d matrices (row[i + j*d] = du_i/dX_j), rows in element order then Gauss
point order, for the material's own elements only; getPotentialEnergy is
(points, 1).
"""
import ast
import math
import re
import weakref

import numpy as np

from . import _abi

# ghost types (aka_common.hh); a single GPU holds no ghost elements
_not_ghost = 0
_ghost = 1
# parameter access flags (ParameterAccessType, parameter_registry.hh): the
# names of the reference, values of this module
_pat_internal = 0x0001
_pat_writable = 0x0010
_pat_readable = 0x0100
_pat_modifiable = _pat_readable | _pat_writable
_pat_parsable = 0x1000
_pat_parsmod = _pat_parsable | _pat_modifiable

# laws the library computes on the device
BUILTIN_LAWS = ("elastic", "neohookean")

_sections = []  # [(law, {key: value})] of the last parseInput
_globals = {}    # its global parameters


_FUNCTIONS = {"max": max, "min": min, "abs": abs, "sqrt": math.sqrt, "exp": math.exp,
              "log": math.log, "sin": math.sin, "cos": math.cos, "tan": math.tan,
              "pow": math.pow, "floor": math.floor, "ceil": math.ceil}
_CONSTANTS = {"pi": math.pi, "e": math.e}


class _Scope:
    """The parameters of a section (raw text), its enclosing scope, and the
    values already evaluated: a name in an expression is looked up here,
    then in the enclosing sections, up to the global parameters (the
    reference's parser resolves them the same way)."""

    def __init__(self, raw, parent=None):
        self.raw, self.parent, self.values, self.busy = raw, parent, {}, set()

    def lookup(self, name):
        scope = self
        while scope is not None:
            if name in scope.raw:
                return scope.value(name)
            scope = scope.parent
        if name in _CONSTANTS:
            return _CONSTANTS[name]
        raise KeyError(name)

    def value(self, name):
        if name == "name":  # a section's name is text, whatever it reads like
            return self.raw[name]
        if name not in self.values:
            if name in self.busy:
                raise KeyError(name)  # a cycle: left as text
            self.busy.add(name)
            try:
                self.values[name] = _evaluate(self.raw[name], self)
            finally:
                self.busy.discard(name)
        return self.values[name]


def _evaluate(text, scope):
    """A parameter's value: an arithmetic expression over numbers, the
    constants pi and e, the parameters in scope and a few functions (max,
    min, sqrt, ...), a vector [a, b, ...] or a matrix [[...], [...]] of
    such expressions, true / false; anything else (a name, a random
    distribution) stays the text it is."""
    t = text.strip()
    if t.lower() in ("true", "false"):
        return t.lower() == "true"
    try:
        tree = ast.parse(t.replace("^", "**"), mode="eval")
    except SyntaxError:
        return t

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return float(node.value)
        if isinstance(node, ast.Name):
            return scope.lookup(node.id) if scope is not None else _CONSTANTS[node.id]
        if isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.USub, ast.UAdd)):
            v = ev(node.operand)
            return -v if isinstance(node.op, ast.USub) else v
        if isinstance(node, ast.BinOp):
            a, b = ev(node.left), ev(node.right)
            ops = {ast.Add: lambda: a + b, ast.Sub: lambda: a - b, ast.Mult: lambda: a * b,
                   ast.Div: lambda: a / b, ast.Pow: lambda: a ** b, ast.Mod: lambda: a % b}
            if type(node.op) in ops:
                return ops[type(node.op)]()
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Name)
                and node.func.id in _FUNCTIONS and not node.keywords):
            return float(_FUNCTIONS[node.func.id](*[ev(a) for a in node.args]))
        if isinstance(node, ast.List):
            return [ev(e) for e in node.elts]
        raise ValueError("not an arithmetic expression")

    try:
        v = ev(tree)
    except (KeyError, ValueError, TypeError, ZeroDivisionError, OverflowError):
        return t
    if isinstance(v, (float, list)) and not isinstance(v, bool):
        return v
    return t


def _value(text):
    """A value with no parameters in scope."""
    return _evaluate(text, None)


_OPEN = re.compile(r"([A-Za-z_]\w*)(?:[ \t]+([A-Za-z_][\w:.-]*))?(?:[ \t]+([A-Za-z_][\w:.-]*))?"
                   r"[ \t\r\n]*\[")
_KEY = re.compile(r"([A-Za-z_]\w*)[ \t]*=[ \t]*")


def parse_input_text(text):
    """The sections of an Akantu input file (Parser::parse, src/io/parser/):
    `type [name [option]] [ ... ]` sections nested at will, `key = value`
    parameters in them and at the top level (the global section), `#`
    comments, a value running to the end of its line (or the closing bracket
    of its section; `\\` continues it on the next line, brackets spanning
    lines do too), evaluated as _evaluate says with names resolved from the
    innermost section out to the global parameters. Keeps the material
    sections (returned, and for the models created after it) and the global
    parameters (input_parameters). Replaces what an earlier call read."""
    global _sections, _globals
    lines = [line.split("#", 1)[0] for line in text.splitlines()]
    body = "\n".join(lines).replace("\\\n", " ")
    root = ("global", "", "", {}, [])  # kind, name, option, raw params, children
    stack = [root]
    pos, n = 0, len(body)
    while True:
        while pos < n and body[pos].isspace():
            pos += 1
        if pos >= n:
            break
        if body[pos] == "]":
            if len(stack) == 1:
                raise ValueError("unbalanced ']' in the input")
            sec = stack.pop()
            if sec[0] == "material" and not sec[1]:
                raise ValueError("material section without a law")
            stack[-1][4].append(sec)
            pos += 1
            continue
        m = _KEY.match(body, pos)
        if m:
            start = end = m.end()
            depth = 0
            while end < n:
                ch = body[end]
                if ch == "[":
                    depth += 1
                elif ch == "]":
                    if depth == 0:
                        break  # the section's closing bracket
                    depth -= 1
                elif ch == "\n" and depth == 0:
                    break
                end += 1
            if depth:
                raise ValueError("unterminated value of '%s'" % m.group(1))
            stack[-1][3][m.group(1)] = " ".join(body[start:end].split())
            pos = end
            continue
        m = _OPEN.match(body, pos)
        if m:
            stack.append((m.group(1), m.group(2) or "", m.group(3) or "", {}, []))
            pos = m.end()
            continue
        line = body[pos:].split("\n", 1)[0]
        raise ValueError("cannot read the input at: %r" % line)
    if len(stack) > 1:
        raise ValueError("unterminated section '%s %s'" % stack[-1][:2])
    found = []

    def walk(sec, parent):
        scope = _Scope(sec[3], parent)
        if sec[0] == "material":
            found.append((sec[1], {k: scope.value(k) for k in sec[3]}))
        for child in sec[4]:
            walk(child, scope)
        return scope

    top = walk(root, None)
    _globals = {k: top.value(k) for k in root[3]}
    _sections = found
    return list(found)


def input_parameters():
    """The global parameters of the last parseInput (Parser::getParameter),
    evaluated."""
    return dict(_globals)


def parseInput(input_file):
    """aka.parseInput (py_parser.cc): reads the material sections of an
    input file for the models created after it."""
    with open(input_file) as f:
        return parse_input_text(f.read())


def input_sections():
    return list(_sections)


class MaterialFactory:
    """aka.MaterialFactory (material.hh:59, 670-691): the allocators of the
    laws written in Python, by law name."""
    _instance = None

    def __init__(self):
        self._allocators = {}

    @classmethod
    def getInstance(cls):
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    def registerAllocator(self, law, allocator):
        """allocator(dim, law, model, material_id) returns the Material."""
        self._allocators[law] = allocator

    def isRegistered(self, law):
        return law in self._allocators

    def allocate(self, law, dim, model, material_id):
        if law not in self._allocators:
            raise KeyError("no material law '%s': not built in (%s) and not registered with "
                           "MaterialFactory" % (law, ", ".join(BUILTIN_LAWS)))
        mat = self._allocators[law](dim, law, model, material_id)
        if not isinstance(mat, Material):
            raise TypeError("the allocator of '%s' did not return a Material" % law)
        return mat


class _InternalField:
    """An internal of the material (InternalField, internal_field.hh): one
    array of nb_component values per quadrature point of the material."""

    def __init__(self, material, nb_component):
        self._material = material
        self.nb_component = int(nb_component)
        self.array = None

    def allocate(self, npoints):
        if self.array is None or self.array.shape[0] != npoints:
            self.array = np.zeros((npoints, self.nb_component))

    def __call__(self, type, ghost_type=_not_ghost):
        self._material._check(type, ghost_type)
        return self.array


class Material:
    """Base of a material law written in Python (py_material.cc: the Python
    side of Material). Subclass it, register parameters in __init__ and
    override computeStress(el_type, ghost_type); computePotentialEnergy and
    getPushWaveSpeed as the reference's Python materials do."""

    def __init__(self, model, _id):
        # the model holds its laws: a weak reference back avoids a cycle that
        # would delay freeing the model's device memory
        self._model = weakref.ref(model) if model is not None else None
        self.id = _id
        self.name = str(_id)
        self._params = {}
        self._docs = {}
        self._internals = {}
        self._el_type = None
        self._elements = None
        self._npoints = 0
        self._grad_u = self._stress = self._energy = None
        self.registerParamReal("rho", _pat_readable | _pat_parsable, "Density")

    # -- parameters (ParameterRegistry, py_parser.cc) ----------------------
    def registerParamReal(self, *args):
        """registerParamReal(name, type, description) or
        registerParamReal(default, name, type, description)."""
        if args and isinstance(args[0], str):
            name, default = args[0], 0.0
            rest = args[1:]
        else:
            default, name = float(args[0]), args[1]
            rest = args[2:]
        self._params.setdefault(name, float(default))
        self._docs[name] = rest[1] if len(rest) > 1 else ""

    def getReal(self, name):
        if name not in self._params:
            raise KeyError("parameter '%s' is not registered" % name)
        return float(self._params[name])

    def setReal(self, name, value):
        if name not in self._params:
            raise KeyError("parameter '%s' is not registered" % name)
        self._params[name] = float(value)

    def getModel(self):
        return self._model() if self._model is not None else None

    # -- the fields of the material's quadrature points --------------------
    def _check(self, el_type, ghost_type):
        if ghost_type != _not_ghost:
            raise ValueError("a single GPU holds no ghost elements")
        if self._el_type is not None and el_type != self._el_type:
            raise ValueError("the material has no elements of type %r" % (el_type,))

    def getGradU(self, el_type, ghost_type=_not_ghost):
        self._check(el_type, ghost_type)
        return self._grad_u

    def getStress(self, el_type, ghost_type=_not_ghost):
        self._check(el_type, ghost_type)
        return self._stress

    def getPotentialEnergy(self, el_type):
        self._check(el_type, _not_ghost)
        return self._energy

    def registerInternal(self, name, nb_component):
        f = _InternalField(self, nb_component)
        self._internals[name] = f
        if self._elements is not None:
            f.allocate(self._npoints)

    @property
    def internals(self):
        return dict(self._internals)

    @property
    def element_filter(self):
        """Callable (type, ghost_type) -> indices of the material's elements."""
        return self.getElementFilter

    def getElementFilter(self, type, ghost_type=_not_ghost):
        self._check(type, ghost_type)
        return self._elements

    # -- to override --------------------------------------------------------
    def initMaterial(self):
        """Allocates the internals of the material's quadrature points; an
        override calls it (super().initMaterial())."""
        for f in self._internals.values():
            f.allocate(self._npoints)

    def computeStress(self, el_type, ghost_type=_not_ghost):
        raise NotImplementedError("computeStress is not implemented by %s"
                                  % type(self).__name__)

    def computePotentialEnergy(self, el_type):
        raise NotImplementedError("computePotentialEnergy is not implemented by %s"
                                  % type(self).__name__)

    def getPushWaveSpeed(self, element):
        """sqrt((lambda + 2 mu) / rho) from the registered E and nu, when
        the law registers them; a law with other parameters overrides it."""
        if "E" not in self._params or "nu" not in self._params:
            raise NotImplementedError("%s registers no E and nu: override getPushWaveSpeed"
                                      % type(self).__name__)
        E, nu, rho = self.getReal("E"), self.getReal("nu"), self.getReal("rho")
        lam = nu * E / ((1 + nu) * (1 - 2 * nu))
        mu = E / (2 * (1 + nu))
        return float(np.sqrt((lam + 2 * mu) / rho))

    # -- set up by the model -------------------------------------------------
    def _attach(self, el_type, elements, nqp, dim):
        self._el_type = el_type
        self._elements = np.asarray(elements, dtype=np.int64)
        self._npoints = len(self._elements) * nqp
        self._grad_u = np.zeros((self._npoints, dim * dim))
        self._stress = np.zeros((self._npoints, dim * dim))
        self._energy = np.zeros((self._npoints, 1))


class MeshDataMaterialSelectorString:
    """MeshDataMaterialSelector<std::string>("physical_names", model)
    (material_selector.hh:151, material_selector_tmpl.hh): an element whose
    physical group (`$PhysicalNames`) names a material of the model takes
    that material, any other element the fallback (material 0 unless
    setFallback says otherwise)."""

    def __init__(self, name, model, first_index=1):
        if name != "physical_names":
            raise ValueError("mesh data '%s': the meshes here carry physical_names only" % name)
        self.model = model
        self.first_index = first_index
        self.fallback = 0

    def setFallback(self, fallback):
        self.fallback = int(fallback)

    def select(self, material_names):
        """The material index of every element, for materials with these
        names in model order."""
        mesh = self.model.mesh
        index = {n: k for k, n in enumerate(material_names)}
        em = np.full(mesh.getNbElement(), self.fallback, dtype=np.uint32)
        for group, elements in mesh.element_groups.items():
            if group in index:
                em[np.asarray(elements, dtype=np.int64)] = index[group]
        return em


def law_from_section(law, params, index, dim, model):
    """The Material of a `material <law> [ ... ]` section written in
    Python: allocated by its factory, its registered parameters set from the
    section (an unregistered one is an error, as in the reference's parser)."""
    mid = str(params.get("name", "%s_%d" % (law, index)))
    mat = MaterialFactory.getInstance().allocate(law, dim, model, mid)
    mat.name = mid
    for key, value in params.items():
        if key in ("name", "finite_deformation"):
            continue
        if key not in mat._params:
            raise KeyError("material '%s': parameter '%s' is not registered by %s"
                           % (mid, key, type(mat).__name__))
        mat.setReal(key, value)
    mat.finite_deformation = bool(params.get("finite_deformation", False))
    return mat


class LawBridge:
    """The Python laws of one model: each law's quadrature points (rows of
    the model-wide quadrature fields), the per-step copies between the
    device fields and the laws' host arrays, and the potential energy from
    the laws' energy densities."""

    def __init__(self, laws, element_material, el_type, nqp, dim):
        self.laws = list(laws)
        self.el_type, self.nqp, self.dim = el_type, nqp, dim
        em = np.asarray(element_material, dtype=np.int64)
        self.rows = []
        for k, law in enumerate(self.laws):
            elements = np.nonzero(em == k)[0]
            law._attach(el_type, elements, nqp, dim)
            self.rows.append((elements[:, None] * nqp + np.arange(nqp)[None, :]).reshape(-1))
        self.npoints = len(em) * nqp
        self.stepped = False

    def stresses(self, grad_u, stress):
        """grad_u, stress: the model's (E*q, d, d) [k, i, j] torch views of
        the column-major device fields. Every law gets its points' gradients
        and writes their stresses; the stresses go back to the device."""
        import torch
        n, d = self.npoints, self.dim
        # the column-major storage: (E*q, d*d), row[i + j*d]
        g = grad_u.transpose(1, 2).reshape(n, d * d).cpu().numpy()
        s = np.zeros((n, d * d))
        for law, rows in zip(self.laws, self.rows):
            law._grad_u[...] = g[rows]
            law.computeStress(self.el_type, _not_ghost)
            s[rows] = law._stress
        stress.transpose(1, 2).reshape(n, d * d).copy_(torch.from_numpy(s))
        self.stepped = True

    def potential_energy(self, weights):
        """sum over the laws' points of the energy density (their
        computePotentialEnergy, at the state of the last step) times the
        point's w det J (Material::getEnergy, material.cc:743-757)."""
        if not self.stepped:
            raise RuntimeError("the potential energy of a Python law needs a step first "
                               "(its stresses are those of the last step)")
        total = 0.0
        for law, rows in zip(self.laws, self.rows):
            law._energy[...] = 0.0
            law.computePotentialEnergy(self.el_type)
            total += float(np.dot(law._energy[:, 0], weights[rows]))
        return total


def qp_weights(mesh):
    """w_q det J_q of every quadrature point, element order then point
    order (the library's user-material point order: hexahedron point q at
    (+-g, +-g, +-g), g = 1/sqrt(3), bit 0 of q for x, bit 1 for y, bit 2 for
    z; one point for the simplices), from the mesh's coordinates."""
    X = np.asarray(mesh.nodes, dtype=np.float64)
    conn = np.asarray(mesh.connectivity, dtype=np.int64)
    t = mesh.element_type
    if t == _abi.SEGMENT_2:
        return X[conn[:, 1], 0] - X[conn[:, 0], 0]
    if t == _abi.TRIANGLE_3:
        J = np.stack([X[conn[:, 1]] - X[conn[:, 0]], X[conn[:, 2]] - X[conn[:, 0]]], axis=1)
        return 0.5 * np.linalg.det(J)
    if t == _abi.TETRAHEDRON_4:
        J = np.stack([X[conn[:, a]] - X[conn[:, 0]] for a in (1, 2, 3)], axis=1)
        return np.linalg.det(J) / 6.0
    sx = np.array([-1, 1, 1, -1, -1, 1, 1, -1], dtype=np.float64)
    sy = np.array([-1, -1, 1, 1, -1, -1, 1, 1], dtype=np.float64)
    sz = np.array([-1, -1, -1, -1, 1, 1, 1, 1], dtype=np.float64)
    g = 1.0 / np.sqrt(3.0)
    Xe = X[conn]  # (E, 8, 3)
    out = np.empty((len(conn), 8))
    for q in range(8):
        cx, cy, cz = (g if q & 1 else -g), (g if q & 2 else -g), (g if q & 4 else -g)
        ax, ay, az = 1 + sx * cx, 1 + sy * cy, 1 + sz * cz
        dN = np.stack([0.125 * sx * ay * az, 0.125 * sy * ax * az, 0.125 * sz * ax * ay])  # (3, 8)
        J = np.einsum("ka,eaj->ekj", dN, Xe)
        out[:, q] = np.linalg.det(J)  # weight 1 per point
    return out.reshape(-1)
