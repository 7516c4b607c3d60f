"""A CPU restatement of the reference's law solver, over the reference's IR JSON. Test infrastructure only.

It evaluates a law the way the reference's CPU solver does — every whole-lattice op in double, stored as float32
between ops (src/field/Law.cpp:757-1468), all-zero results turned into the scalar 0 (`settle`, Law.cpp:554-563), the
cheaper factor of a product first (Law.cpp:818-830) — and steps it as its Solver does: terms in order (Lie splitting),
substeps from max_dt capped at 4096, gather-then-apply with `delta = float(value * sub_dt)`, `T += delta` in float,
the conserved totals in double and the range contract after each term (src/field/Solver.cpp:273-461).

Input: the IR JSON the reference's lawc writes (and libfe_b200's fe_law_ir_json writes identically). Fields are numpy
arrays shaped (nz, ny, nx). Pinned bit for bit against the reference's own solver in tests/test_oracle_pin.py.
"""
import json
import math
import os

import numpy as np

F32 = np.float32


class Law:
    def __init__(self, ir_json):
        ir = json.loads(ir_json) if isinstance(ir_json, str) else ir_json
        self.ir = ir
        self.insts = ir["insts"]
        self.fields = [f["name"] for f in ir["fields"]]
        self.decls = ir["fields"]
        self.params = [p["value"] for p in ir["params"]]
        self.param_names = [p["name"] for p in ir["params"]]
        self.terms = ir["terms"]
        self.derives = ir["derives"]
        self._cost = [None] * len(self.insts)
        self.nets = [Net(n) for n in ir.get("nets", [])]

    def cost(self, i):
        """Subtree size, everything inlined (the reference's node cost, Law.cpp:1518-1521)."""
        if self._cost[i] is None:
            self._cost[i] = 1 + sum(self.cost(a) for a in self.insts[i]["args"])
        return self._cost[i]


class Net:
    """A law's net with its parameters: its weight file if there is one (relative to the working directory, as for the
    reference), else the untrained start (src/field/nn/Net.cpp:241-333)."""

    def __init__(self, decl):
        self.name = decl["name"]
        self.sizes = list(decl["sizes"])
        self.act = decl["act"]
        self.out_scale = np.float32(1.0)
        self.shift = np.zeros(self.sizes[0], F32)
        self.scale = np.ones(self.sizes[0], F32)
        self.weights = self._init()
        if os.path.exists(decl["file"]):
            self._load(decl["file"])

    def offset(self, layer):
        return sum((self.sizes[l] + 1) * self.sizes[l + 1] for l in range(layer))

    def _init(self, seed=0):
        mask = (1 << 64) - 1

        def fin(h):
            h ^= h >> 33
            h = (h * 0xFF51AFD7ED558CCD) & mask
            h ^= h >> 33
            h = (h * 0xC4CEB9FE1A85EC53) & mask
            h ^= h >> 33
            return h
        w = np.zeros(self.offset(len(self.sizes) - 1), F32)
        h = 1469598103934665603 ^ seed
        for c in self.name.encode():
            h = ((h ^ c) * 1099511628211) & mask
        for l in range(len(self.sizes) - 2):
            ni, no = self.sizes[l], self.sizes[l + 1]
            limit = np.sqrt(F32(6.0) / F32(ni + no), dtype=F32)
            base = self.offset(l)
            for k in range(ni * no):
                r = fin((h + l * 0x9E3779B97F4A7C15 + k) & mask)
                u = F32((r >> 11) * (1.0 / 9007199254740992.0))
                w[base + k] = (F32(2.0) * u - F32(1.0)) * limit
        return w

    def _load(self, path):
        words = open(path).read().split()
        section, i = None, 0
        sizes, shift, scale, weights = [], [], [], []
        while i < len(words):
            w = words[i]
            i += 1
            if w == "net":
                i += 1
            elif w == "act":
                i += 1
                section = None
            elif w == "out_scale":
                self.out_scale = F32(float(words[i]))
                i += 1
                section = None
            elif w in ("sizes", "in_shift", "in_scale", "weights"):
                section = w
            else:
                {"sizes": sizes, "in_shift": shift, "in_scale": scale, "weights": weights}[section].append(float(w))
        assert [int(s) for s in sizes] == self.sizes, path
        self.weights = np.array(weights, F32)
        self.shift = np.zeros(self.sizes[0], F32)
        self.shift[:len(shift)] = shift
        self.scale = np.ones(self.sizes[0], F32)
        self.scale[:len(scale)] = scale

    def _activate(self, v):
        if self.act == "tanh":
            return np.tanh(v.astype(np.float64)).astype(F32)
        if self.act == "relu":
            return np.where(v > 0, v, F32(0.0)).astype(F32)
        if self.act == "silu":
            return (v / (F32(1.0) + np.exp(-v.astype(np.float64)).astype(F32))).astype(F32)
        return v

    def forward(self, x):
        """x: (cells, inputs) float32 -> (cells, outputs) float32, in the reference's float order."""
        h = ((x.astype(F32) - self.shift) * self.scale).astype(F32)
        layers = len(self.sizes) - 1
        for l in range(layers):
            ni, no = self.sizes[l], self.sizes[l + 1]
            w = self.weights[self.offset(l):self.offset(l) + ni * no].reshape(no, ni)
            b = self.weights[self.offset(l) + ni * no:self.offset(l) + ni * no + no]
            out = np.empty((h.shape[0], no), F32)
            for o in range(no):
                acc = np.full(h.shape[0], b[o], F32)
                for i in range(ni):
                    acc = (acc + (w[o, i] * h[:, i]).astype(F32)).astype(F32)
                out[:, o] = acc
            h = self._activate(out) if l + 1 < layers else out
        return (h * self.out_scale).astype(F32)


def _settle(a):
    a = np.asarray(a, dtype=F32)
    return 0.0 if not np.any(a != 0) else a


def _is_scalar(v):
    return not isinstance(v, np.ndarray)


def _uniform(v):
    return _is_scalar(v) or bool(np.all(v == v.reshape(-1)[0]))


class Evaluator:
    """One gather: every value of the pre-state computed once (the reference's epoch sharing)."""

    def __init__(self, law, fields, zero, h, dt, keep=None):
        self.law = law
        self.keep = keep if keep is not None else {}  # what distance and poisson keep between evaluations
        self.fields = fields
        self.zero = zero
        self.h = h
        self.dt = dt
        self.memo = {}
        self.shape = next(iter(fields.values())).shape if fields else (1, 1, 1)

    def __call__(self, i):
        if i not in self.memo:
            self.memo[i] = self._eval(i)
        return self.memo[i]

    def _arr(self, v):
        return np.full(self.shape, v, dtype=np.float64) if _is_scalar(v) else v.astype(np.float64)

    def _eval(self, i):
        ins = self.law.insts[i]
        op = ins["op"]
        a = ins["args"]
        h = self.h
        nz, ny, nx = self.shape
        if op == "const":
            return float(ins["number"])
        if op == "param":
            return float(self.law.params[ins["index"]])
        if op == "h":
            return float(h)
        if op == "dt":
            return float(self.dt)
        if op == "field":
            f = self.law.fields[ins["index"]]
            return 0.0 if self.zero[f] else self.fields[f]
        if op == "rim":
            z, y, x = np.indices(self.shape)
            r = ((x == 0) | (y == 0) | (z == 0) | (x == nx - 1) | (y == ny - 1) | (z == nz - 1)).astype(F32)
            return _settle(r)
        unary = {
            "neg": lambda v: -v, "abs": np.abs, "sqrt": lambda v: np.sqrt(np.maximum(0.0, v)),
            "exp": lambda v: np.exp(np.minimum(v, 80.0)), "log": lambda v: np.log(np.maximum(v, 1e-30)),
            "step": lambda v: np.where(v > 0.0, 1.0, 0.0), "pos": lambda v: np.maximum(v, 0.0),
        }
        if op in unary:
            v = self(a[0])
            if _is_scalar(v):
                return float(unary[op](np.float64(v)))
            with np.errstate(all="ignore"):
                return _settle(unary[op](v.astype(np.float64)).astype(F32))
        if op == "mul":
            # The cheaper factor first; a scalar zero ends it without looking at the other (Law.cpp:818-830).
            swap = self.law.cost(a[1]) < self.law.cost(a[0])
            first, second = (a[1], a[0]) if swap else (a[0], a[1])
            fa = self(first)
            if _is_scalar(fa) and fa == 0.0:
                return 0.0
            fb = self(second)
            if _is_scalar(fb) and fb == 0.0:
                return 0.0
            x, y = (fb, fa) if swap else (fa, fb)
            if _is_scalar(x) and _is_scalar(y):
                return x * y
            with np.errstate(all="ignore"):
                return _settle((np.float64(x) if _is_scalar(x) else x.astype(np.float64)) *
                               (np.float64(y) if _is_scalar(y) else y.astype(np.float64)))
        binary = {
            "add": lambda p, q: p + q, "sub": lambda p, q: p - q,
            "div": lambda p, q: np.where(q == 0.0, 0.0, p / np.where(q == 0.0, 1.0, q)),
            "pow": lambda p, q: np.power(p, q), "min": np.minimum, "max": np.maximum,
        }
        if op in binary:
            x, y = self(a[0]), self(a[1])
            with np.errstate(all="ignore"):
                if _is_scalar(x) and _is_scalar(y):
                    return float(binary[op](np.float64(x), np.float64(y)))
                xx = np.float64(x) if _is_scalar(x) else x.astype(np.float64)
                yy = np.float64(y) if _is_scalar(y) else y.astype(np.float64)
                return _settle(np.asarray(binary[op](xx, yy)).astype(F32))
        if op == "clamp":
            x, lo, hi = self(a[0]), self(a[1]), self(a[2])
            if all(_is_scalar(v) for v in (x, lo, hi)):
                return float(min(max(x, lo), max(lo, hi)))
            xx, ll, hh = self._arr(x), self._arr(lo), self._arr(hi)
            return _settle(np.minimum(np.maximum(xx, ll), np.maximum(ll, hh)).astype(F32))
        if op == "shift":
            v = self(a[0])
            if _is_scalar(v):
                return v
            dx, dy, dz = ins["offset"]
            zi = np.clip(np.arange(nz) + dz, 0, nz - 1)
            yi = np.clip(np.arange(ny) + dy, 0, ny - 1)
            xi = np.clip(np.arange(nx) + dx, 0, nx - 1)
            return _settle(v[zi][:, yi][:, :, xi])
        if op in ("shift_t", "gx_t", "gy_t", "gz_t"):
            return self._transposed(op, ins, self._arr(self(a[0])))
        if op in ("lap", "gx", "gy", "gz"):
            v = self(a[0])
            if _uniform(v):
                return 0.0
            return _settle(self._stencil(op, v))
        if op == "diffuse":
            return self._diffuse(self(a[0]), self(a[1]))
        if op == "adv":
            return self._adv(self(a[0]), self(a[1]), self(a[2]), self(a[3]))
        if op == "tridiag":
            return self._tridiag(ins["index"], *(self(x) for x in a))
        if op in ("maxof", "minof", "sumof"):
            v = self(a[0])
            if _is_scalar(v):
                return v * (nx * ny * nz) if op == "sumof" else v
            flat = v.reshape(-1).astype(np.float64)
            if op == "sumof":
                acc = 0.0
                for x in flat:  # in order, in double (Law.cpp:1449-1466)
                    acc += x
                return acc
            return float(flat.max() if op == "maxof" else flat.min())
        if op in ("fall", "spread", "topple"):
            return getattr(self, "_" + op)(*(self(x) for x in a))
        if op == "mlp":
            net = self.law.nets[ins["index"]]
            xs = [self(x) for x in a]
            if all(_is_scalar(v) for v in xs):
                return float(net.forward(np.array([[F32(v) for v in xs]], F32))[0, 0])
            x = np.stack([self._arr(v).astype(F32).reshape(-1) for v in xs], axis=1)
            return _settle(net.forward(x)[:, 0].reshape(self.shape))
        if op == "flux":
            return self._flux(self.law.nets[ins["index"]], [self(x) for x in a[:-2]], self.law.insts[a[-2]]["number"],
                              self.law.insts[a[-1]]["number"])
        if op == "ldiffuse":
            return self._ldiffuse(self.law.nets[ins["index"]], self(a[0]), self(a[1]))
        if op == "distance":
            return self._distance(i, self._arr(self(a[0])).astype(F32))
        if op == "poisson":
            return self._poisson(i, self._arr(self(a[0])).astype(F32), int(ins["iterations"]))
        raise NotImplementedError(f"the oracle does not restate '{op}'")

    # ---- the net ops' faces (Law.cpp:672-738, 1335-1438) -------------------------------------------------------------
    def _faces_to_cells(self, wide):
        """wide[0], [1], [2]: the flux from each cell through its +x, +y, +z face (0 where there is none); the cell's
        gain over h."""
        out = np.zeros(self.shape, F32)
        for a, axis in enumerate((2, 1, 0)):  # x, y, z: each its lower face's in, then its upper face's out
            lower = np.zeros(self.shape, F32)
            sl_dst = [slice(None)] * 3
            sl_src = [slice(None)] * 3
            sl_dst[axis], sl_src[axis] = slice(1, None), slice(None, -1)
            lower[tuple(sl_dst)] = wide[a][tuple(sl_src)]
            out = (out + lower).astype(F32)
            out = (out - wide[a]).astype(F32)
        return _settle((out / F32(self.h)).astype(F32))

    def _pairs(self, axis):
        """Index arrays (i, j) of every face along an axis, i the lower cell."""
        n = self.shape[axis]
        idx = np.arange(int(np.prod(self.shape))).reshape(self.shape)
        sl_i = [slice(None)] * 3
        sl_j = [slice(None)] * 3
        sl_i[axis], sl_j[axis] = slice(None, n - 1), slice(1, None)
        return idx[tuple(sl_i)], idx[tuple(sl_j)], tuple(sl_i)

    def _flux(self, net, vals, lo, hi):
        if all(_uniform(v) for v in vals):
            return 0.0
        arrs = [self._arr(v).astype(F32).reshape(-1) for v in vals]
        m = len(arrs)
        dt = self.dt
        per = F32(0.999 * self.h / (6.0 * dt)) if dt > 0 else None
        wide = []
        for axis in (2, 1, 0):
            w = np.zeros(self.shape, F32)
            i, j, sl = self._pairs(axis)
            if i.size:
                i, j = i.reshape(-1), j.reshape(-1)
                xi = np.stack([a[i] for a in arrs], axis=1)
                xj = np.stack([a[j] for a in arrs], axis=1)
                gij = net.forward(np.concatenate([xi, xj], axis=1))[:, 0]
                gji = net.forward(np.concatenate([xj, xi], axis=1))[:, 0]
                r = (F32(0.5) * (gij - gji).astype(F32)).astype(F32)
                if per is not None:
                    fi, fj = xi[:, 0], xj[:, 0]
                    pos, neg = r > 0, r < 0
                    if lo > -1e29:
                        r = np.where(pos, np.minimum(r, np.maximum(F32(0), ((fi - F32(lo)) * per).astype(F32))), r)
                    if hi < 1e29:
                        r = np.where(pos, np.minimum(r, np.maximum(F32(0), ((F32(hi) - fj) * per).astype(F32))), r)
                    if lo > -1e29:
                        r = np.where(neg, np.maximum(r, -np.maximum(F32(0), ((fj - F32(lo)) * per).astype(F32))), r)
                    if hi < 1e29:
                        r = np.where(neg, np.maximum(r, -np.maximum(F32(0), ((F32(hi) - fi) * per).astype(F32))), r)
                w[sl] = r.astype(F32).reshape(w[sl].shape)
            wide.append(w)
        return self._faces_to_cells(wide)

    def _ldiffuse(self, net, k, f):
        if _uniform(f):
            return 0.0
        F = self._arr(f).astype(F32)
        K = self._arr(k)
        dt = F32(self.dt)
        h = F32(self.h)
        wide = []
        for axis in (2, 1, 0):
            n = self.shape[axis]
            w = np.zeros(self.shape, F32)
            if n > 1:
                q = np.arange(n)
                im = np.where(q > 0, q - 1, q)[:n - 1]
                jp = np.where(q + 2 < n, q + 2, q + 1)[:n - 1]
                take = lambda a, idx: np.take(a, idx, axis=axis)
                win = [take(F, im), take(F, q[:n - 1]), take(F, q[1:]), take(F, jp)]
                ka = take(K, q[:n - 1]).astype(np.float64)
                kb = take(K, q[1:]).astype(np.float64)
                s = ka + kb
                kf = np.where(s > 0, 2.0 * ka * kb / np.where(s > 0, s, 1.0), 0.0).astype(F32)

                def raw(wv):
                    centre = (F32(0.5) * (wv[1] + wv[2]).astype(F32)).astype(F32)
                    spread = np.full(centre.shape, F32(1e-6), F32)
                    for a in range(4):
                        spread = np.maximum(spread, np.abs((wv[a] - centre).astype(F32)))
                    x = [((wv[a] - centre).astype(F32) / spread).astype(F32) for a in range(4)]
                    x.append(((kf * dt).astype(F32) / (h * h)).astype(F32))
                    y = net.forward(np.stack([v.reshape(-1) for v in x], axis=1))
                    y = [y[:, a].reshape(centre.shape) for a in range(4)]
                    mean = (F32(0.25) * ((((y[0] + y[1]).astype(F32) + y[2]).astype(F32) + y[3]).astype(F32))).astype(F32)
                    acc = np.zeros(centre.shape, F32)
                    for a, base in enumerate((0.0, -1.0, 1.0, 0.0)):
                        acc = (acc + ((F32(base) + (y[a] - mean).astype(F32)).astype(F32) * wv[a]).astype(F32)).astype(F32)
                    return ((-kf / h).astype(F32) * acc).astype(F32)
                ij = raw(win)
                ji = raw(win[::-1])
                sl = [slice(None)] * 3
                sl[axis] = slice(None, n - 1)
                w[tuple(sl)] = (F32(0.5) * (ij - ji).astype(F32)).astype(F32)
            wide.append(w)
        return self._faces_to_cells(wide)

    # ---- the whole-lattice ops (Law.cpp:1042-1098, 1139-1181) ---------------------------------------------------------
    @staticmethod
    def _squared_distance(feature):
        """Exact squared distance (in cells) of every cell to the nearest cell of `feature`, inf without one: a 1-D
        pass along x, then y, then z, each the least over the axis of (what the previous pass found) + r^2
        (Law.cpp:489-525 computes the same numbers with a lower-envelope pass)."""
        d = np.where(feature, 0.0, np.inf)
        for axis in (2, 1, 0):
            n = d.shape[axis]
            if n == 1:
                continue
            best = d.copy()
            for r in range(1, n):
                rr = float(r * r)
                lo = np.full_like(d, np.inf)
                hi = np.full_like(d, np.inf)
                sl_dst = [slice(None)] * 3
                sl_src = [slice(None)] * 3
                sl_dst[axis], sl_src[axis] = slice(r, None), slice(None, n - r)
                lo[tuple(sl_dst)] = d[tuple(sl_src)]
                sl_dst[axis], sl_src[axis] = slice(None, n - r), slice(r, None)
                hi[tuple(sl_dst)] = d[tuple(sl_src)]
                best = np.minimum(best, np.minimum(lo, hi) + rr)
            d = best
        return d

    def _distance(self, i, a):
        """Signed distance in metres to the surface of {a >= 0.5} (negative inside), the surface half a cell from the
        last solid cell's centre, beyond the lattice open. Recomputed only when a's bits change (Law.cpp:1042-1098)."""
        key = ("distance", i)
        k = a.tobytes()
        if key in self.keep and self.keep[key][0] == k:
            return self.keep[key][1]
        nz, ny, nx = self.shape
        h = self.h
        far = (nx + ny + nz) * h
        inside = a >= 0.5
        any_in, any_out = bool(inside.any()), bool((~inside).any())
        to_in = self._squared_distance(inside) if any_in else None
        to_out = self._squared_distance(~inside) if any_out else None
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        border = np.full(self.shape, np.inf)
        for q, n in ((x, nx), (y, ny), (z, nz)):
            if n > 1:
                border = np.minimum(border, np.minimum(q + 1, n - q).astype(np.float64))
        out_cells = np.minimum(np.sqrt(to_out) if any_out else far / h, border)
        d_in = -(out_cells - 0.5) * h
        d_out = (np.sqrt(to_in) - 0.5) * h if any_in else np.full(self.shape, far)
        out = np.where(inside, d_in, d_out).astype(F32)
        self.keep[key] = (k, out)
        return out

    def _poisson(self, i, s, iterations):
        """`iterations` Jacobi sweeps of lap(phi) = s (phi = 0 beyond the lattice), warm-started from the last answer;
        skipped while s keeps its bits (Law.cpp:1139-1181)."""
        key = ("poisson", i)
        k = s.tobytes()
        phi = self.keep.get(key, (None, np.zeros(self.shape, F32)))
        if phi[0] == k:
            return phi[1]
        phi = phi[1]
        nz, ny, nx = self.shape
        axes = sum(1 for n in (nx, ny, nz) if n > 1)
        denom = 2.0 * max(axes, 1)
        h = self.h
        src = s.astype(np.float64)
        for _ in range(iterations):
            p = phi.astype(np.float64)
            total = np.zeros(self.shape)
            for axis, n in ((2, nx), (1, ny), (0, nz)):
                if n < 2:
                    continue
                lo = np.zeros(self.shape)
                hi = np.zeros(self.shape)
                sl_dst = [slice(None)] * 3
                sl_src = [slice(None)] * 3
                sl_dst[axis], sl_src[axis] = slice(1, None), slice(None, -1)
                lo[tuple(sl_dst)] = p[tuple(sl_src)]
                sl_dst[axis], sl_src[axis] = slice(None, -1), slice(1, None)
                hi[tuple(sl_dst)] = p[tuple(sl_src)]
                total = total + lo
                total = total + hi
            phi = ((total - h * h * src) / denom).astype(F32)
        self.keep[key] = (k, phi)
        return phi

    # ---- stencils (Law.cpp:947-985) ----------------------------------------------------------------------------------
    def _neighbours(self, v):
        nz, ny, nx = self.shape
        x = np.arange(nx)
        y = np.arange(ny)
        z = np.arange(nz)
        xm, xp = np.maximum(x - 1, 0), np.minimum(x + 1, nx - 1)
        ym, yp = np.maximum(y - 1, 0), np.minimum(y + 1, ny - 1)
        zm, zp = np.maximum(z - 1, 0), np.minimum(z + 1, nz - 1)
        return (v[:, :, xm], v[:, :, xp], v[:, ym, :], v[:, yp, :], v[zm], v[zp], (xm, xp, ym, yp, zm, zp))

    def _stencil(self, op, v):
        h = self.h
        d = v.astype(np.float64)
        vxm, vxp, vym, vyp, vzm, vzp, (xm, xp, ym, yp, zm, zp) = self._neighbours(d)
        nz, ny, nx = self.shape
        with np.errstate(all="ignore"):
            if op == "lap":
                out = (vxm + vxp + vym + vyp + vzm + vzp - 6.0 * d) / (h * h)
            elif op == "gx":
                out = (vxp - vxm) / (h * (xp - xm).astype(np.float64))[None, None, :]
            elif op == "gy":
                out = (vyp - vym) / (h * (yp - ym).astype(np.float64))[None, :, None] if ny > 1 else np.zeros(self.shape)
            else:
                out = (vzp - vzm) / (h * (zp - zm).astype(np.float64))[:, None, None] if nz > 1 else np.zeros(self.shape)
        return np.where(np.isfinite(out), out, 0.0).astype(F32)

    @staticmethod
    def _run(n, d):
        """For each cell j along an axis of n cells, the cells i with clamp(i + d) = j: one run lo..hi (Law.cpp:876-882)."""
        j = np.arange(n)
        lo = np.maximum(np.where(j == 0, 0, j - d), 0)
        hi = np.minimum(np.where(j == n - 1, n - 1, j - d), n - 1)
        return lo, hi

    def _transposed(self, op, ins, v):
        """shift_t and gx_t/gy_t/gz_t, what each cell sent to the cells that read it gathered back, summed in double in
        the reference's loop order (Law.cpp:870-919)."""
        nz, ny, nx = self.shape
        h = self.h
        out = np.zeros(self.shape)
        if op == "shift_t":
            dx, dy, dz = ins["offset"]
            runs = [self._run(n, d) for n, d in ((nz, dz), (ny, dy), (nx, dx))]
            width = [int(np.max(hi - lo + 1)) if len(lo) else 0 for lo, hi in runs]
            for kz in range(max(width[0], 0)):
                zz = runs[0][0] + kz
                okz = zz <= runs[0][1]
                for ky in range(max(width[1], 0)):
                    yy = runs[1][0] + ky
                    oky = yy <= runs[1][1]
                    for kx in range(max(width[2], 0)):
                        xx = runs[2][0] + kx
                        okx = xx <= runs[2][1]
                        ok = okz[:, None, None] & oky[None, :, None] & okx[None, None, :]
                        vals = v[np.clip(zz, 0, nz - 1)][:, np.clip(yy, 0, ny - 1)][:, :, np.clip(xx, 0, nx - 1)]
                        out = out + np.where(ok, vals, 0.0)
            return _settle(out.astype(F32))
        axis = {"gx_t": 2, "gy_t": 1, "gz_t": 0}[op]
        n = self.shape[axis]
        q = np.arange(n)
        span = (np.minimum(q + 1, n - 1) - np.maximum(q - 1, 0)).astype(np.float64)
        shape = [1, 1, 1]
        shape[axis] = n
        with np.errstate(all="ignore"):
            w = np.where(span.reshape(shape) > 0, v / (h * span.reshape(shape)), 0.0)
        for d in (1, -1):
            lo, hi = self._run(n, d)
            for k in range(int(np.max(hi - lo + 1)) if n else 0):
                idx = lo + k
                ok = (idx <= hi).reshape(shape)
                vals = np.take(w, np.clip(idx, 0, n - 1), axis=axis)
                out = out + np.where(ok, vals if d > 0 else -vals, 0.0)
        return _settle(out.astype(F32))

    def _active_planes(self, v):
        nz = self.shape[0]
        flat = np.array([bool(np.all(v[z] == v[z].reshape(-1)[0])) for z in range(nz)])
        level = np.array([v[z].reshape(-1)[0] for z in range(nz)])
        act = np.zeros(nz, bool)
        for z in range(nz):
            m = not flat[z]
            if z > 0:
                m = m or not flat[z - 1] or level[z - 1] != level[z]
            if z + 1 < nz:
                m = m or not flat[z + 1] or level[z + 1] != level[z]
            act[z] = m
        return act

    def _diffuse(self, k, f):
        """Flux form with the harmonic face conductivity, in double (Law.cpp:986-1018)."""
        if _uniform(f):
            return 0.0
        h = self.h
        nz, ny, nx = self.shape
        v = f.astype(np.float64)
        kk = self._arr(k)
        acc = np.zeros(self.shape)
        for axis, n in ((2, nx), (1, ny), (0, nz)):
            for sign in (-1, 1):
                nb = np.roll(v, -sign, axis=axis)
                kb = np.roll(kk, -sign, axis=axis)
                with np.errstate(all="ignore"):
                    kf = np.where(kk + kb > 0.0, 2.0 * kk * kb / np.where(kk + kb > 0.0, kk + kb, 1.0), 0.0)
                idx = np.arange(n) + sign
                valid = ((idx >= 0) & (idx < n))
                shape = [1, 1, 1]
                shape[axis] = n
                acc += np.where(valid.reshape(shape), kf * (nb - v), 0.0)
        out = (acc / (h * h)).astype(F32)
        act = self._active_planes(f)
        out[~act] = 0.0
        return _settle(out)

    def _adv(self, f, u, w, s):
        """Upwind -(u . grad F) (Law.cpp:1019-1040)."""
        if _uniform(f):
            return 0.0
        h = self.h
        v = f.astype(np.float64)
        out = np.zeros(self.shape)
        for axis, speed in ((2, u), (1, w), (0, s)):
            sp = self._arr(speed)
            n = self.shape[axis]
            c = np.indices(self.shape)[axis]
            lo = np.roll(v, 1, axis=axis)
            hi = np.roll(v, -1, axis=axis)
            up = np.where(sp > 0.0, np.where(c > 0, sp * (v - lo) / h, 0.0), np.where(c + 1 < n, sp * (hi - v) / h, 0.0))
            out += up
        return _settle((-out).astype(F32))

    def _tridiag(self, index, lo, di, up, rhs):
        """Thomas' algorithm in double, a line at a time, the edge cell repeating (Law.cpp:1098-1138). index 3 + axis:
        the transposed system (tridiag_x_t, an adjoint op this build adds): below the diagonal the previous cell's up,
        above it the next cell's lo, the edge cells' folded terms on the diagonal."""
        axis = index % 3
        L, D, U, R = (np.moveaxis(self._arr(x), 2 - axis, -1) for x in (lo, di, up, rhs))
        n = L.shape[-1]
        if index >= 3:
            Lt = np.zeros(L.shape)
            Ut = np.zeros(L.shape)
            Dt = D.copy()
            Lt[..., 1:] = U[..., :-1]
            Ut[..., :-1] = L[..., 1:]
            Dt[..., 0] = Dt[..., 0] + L[..., 0]
            Dt[..., n - 1] = Dt[..., n - 1] + U[..., n - 1]
            L, D, U = Lt, Dt, Ut
        c = np.zeros(L.shape)
        d = np.zeros(L.shape)
        for i in range(n):
            a = L[..., i]
            b = D[..., i] + (a if i == 0 else 0.0) + (U[..., i] if i + 1 == n else 0.0)
            m = b if i == 0 else b - a * c[..., i - 1]
            c[..., i] = 0.0 if i + 1 == n else U[..., i] / m
            d[..., i] = (R[..., i] - (0.0 if i == 0 else a * d[..., i - 1])) / m
        x = np.zeros(L.shape, dtype=F32)
        nxt = np.zeros(L.shape[:-1])
        for i in range(n - 1, -1, -1):
            nxt = d[..., i] - c[..., i] * nxt
            x[..., i] = nxt.astype(F32)
        return np.moveaxis(x, -1, 2 - axis)

    # ---- matter ops (Law.cpp:1192-1334) -----------------------------------------------------------------------------
    def _fall(self, f, b, speed):
        nz = self.shape[0]
        if _is_scalar(f) or nz < 2:
            return 0.0
        h = self.h
        fv = f.astype(np.float64)
        bb = self._arr(b)
        sp = self._arr(speed)
        wide = np.zeros(self.shape)
        free = np.clip(1.0 - bb[:-1] - fv[:-1], 0.0, 1.0)
        wide[1:] = np.maximum(0.0, sp[1:]) / h * np.maximum(0.0, fv[1:]) * free
        out = (0.0 - wide).astype(F32)
        out[:-1] = (out[:-1] + wide[1:]).astype(F32)
        return _settle(out)

    def _spread(self, f, b, k):
        if _uniform(f):
            return 0.0
        h = self.h
        fv = f.astype(np.float64)
        bb = self._arr(b)
        kk = self._arr(k)
        nz, ny, nx = self.shape

        def flux(fa, fc, ba, bc, ka, kc, fra, frc):
            r_is_c = fa > fc
            free = np.clip(1.0 - np.where(r_is_c, bc, ba) - np.where(r_is_c, frc, fra), 0.0, 1.0)
            kf = 0.5 * (np.maximum(0.0, ka) + np.maximum(0.0, kc))
            return kf / (h * h) * (fa - fc) * free

        wx = np.zeros(self.shape)
        wy = np.zeros(self.shape)
        wx[:, :, :-1] = flux(fv[:, :, :-1], fv[:, :, 1:], bb[:, :, :-1], bb[:, :, 1:], kk[:, :, :-1], kk[:, :, 1:], fv[:, :, :-1], fv[:, :, 1:])
        wy[:, :-1, :] = flux(fv[:, :-1, :], fv[:, 1:, :], bb[:, :-1, :], bb[:, 1:, :], kk[:, :-1, :], kk[:, 1:, :], fv[:, :-1, :], fv[:, 1:, :])
        out = np.zeros(self.shape, F32)
        out[:, 1:, :] = (out[:, 1:, :] + wy[:, :-1, :]).astype(F32)
        out[:, :, 1:] = (out[:, :, 1:] + wx[:, :, :-1]).astype(F32)
        out = (out - wx).astype(F32)
        out = (out - wy).astype(F32)
        return _settle(out)

    def _topple(self, f, b, rate):
        nz, ny, nx = self.shape
        if _is_scalar(f) or nz < 2:
            return 0.0
        h = self.h
        fv = f.astype(np.float64)
        bb = self._arr(b)
        rr = self._arr(rate)
        room = np.clip(1.0 - bb - fv, 0.0, 1.0)
        wide = np.zeros((4,) + self.shape)
        z, y, x = np.indices(self.shape)
        below_room = np.zeros(self.shape)
        below_room[1:] = room[:-1]
        can = (fv > 0.0) & (z > 0) & ~(below_room > 0.01)
        shifts = [(-1, 0), (1, 0), (0, -1), (0, 1)]
        for s, (sx, sy) in enumerate(shifts):
            jx = x + sx
            jy = y + sy
            inside = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny)
            jxc = np.clip(jx, 0, nx - 1)
            jyc = np.clip(jy, 0, ny - 1)
            zc = np.maximum(z - 1, 0)
            rj = room[z, jyc, jxc]
            rjb = room[zc, jyc, jxc]
            w = 0.25 * np.maximum(0.0, rr) / h * fv * np.minimum(rj, rjb)
            wide[s] = np.where(can & inside, w, 0.0)
        out = np.zeros(self.shape)
        for s in range(4):
            out -= wide[s]
        up = np.zeros((4,) + self.shape)
        up[:, :-1] = wide[:, 1:]
        add = np.zeros(self.shape)
        # cell (x, y, z) gains what slid off (x+1, y, z+1) going -x, (x-1, y, z+1) going +x, (x, y+1, z+1) going -y,
        # (x, y-1, z+1) going +y, in that order.
        t = np.zeros(self.shape)
        t[:, :, :-1] = up[0][:, :, 1:]
        add = add + t
        t = np.zeros(self.shape)
        t[:, :, 1:] = up[1][:, :, :-1]
        add = add + t
        t = np.zeros(self.shape)
        t[:, :-1, :] = up[2][:, 1:, :]
        add = add + t
        t = np.zeros(self.shape)
        t[:, 1:, :] = up[3][:, :-1, :]
        add = add + t
        out = out + add
        return _settle(out.astype(F32))


class Solver:
    """Steps a law like the reference's CPU Solver (src/field/Solver.cpp:273-461)."""

    MAX_SUBSTEPS = 4096

    def __init__(self, law, shape, h):
        self.law = law
        self.h = h
        self.shape = shape
        self.fields = {}
        for d in law.decls:
            self.fields[d["name"]] = np.full(shape, F32(d["init"]), dtype=F32)
        self.violations = []
        self.substeps = [1] * len(law.terms)
        self.keep = {}  # distance's and poisson's answers and the inputs they were solved for

    def _zero(self):
        return {k: not np.any(v != 0) for k, v in self.fields.items()}

    def step(self, dt):
        self.violations = []
        for t, term in enumerate(self.law.terms):
            self._integrate(t, term, dt)
        for d in self.law.derives:
            ev = Evaluator(self.law, self.fields, self._zero(), self.h, 0.0, self.keep)
            target = self.law.fields[d["equations"][0][0]]
            v = ev(d["equations"][0][1])
            old = self.fields[target].astype(np.float64) if d["accumulate"] else 0.0
            self.fields[target] = (old + (np.float64(v) if _is_scalar(v) else v.astype(np.float64))).astype(F32) * np.ones(self.shape, F32)

    def _integrate(self, t, term, dt):
        law = self.law
        self.substeps[t] = 1
        count = 1
        if term["max_dt"] >= 0:
            ev = Evaluator(law, self.fields, self._zero(), self.h, 0.0, self.keep)
            limit = ev(term["max_dt"])
            if _is_scalar(limit) and limit > 0.0 and math.isfinite(limit) and dt > limit:
                wanted = math.ceil(dt / limit)
                if wanted > self.MAX_SUBSTEPS:
                    self.violations.append(("substep-cap", t))
                    count = self.MAX_SUBSTEPS
                else:
                    count = int(wanted)
        self.substeps[t] = count
        sub_dt = dt / count
        before = None
        touched = False
        for _ in range(count):
            ev = Evaluator(law, self.fields, self._zero(), self.h, sub_dt, self.keep)
            deltas = []
            for target, value in term["equations"]:
                v = ev(value)
                if _is_scalar(v) and v == 0.0:
                    deltas.append(None)
                    continue
                if _is_scalar(v):
                    deltas.append(np.full(self.shape, F32(v * sub_dt), dtype=F32))
                else:
                    deltas.append((v.astype(np.float64) * sub_dt).astype(F32))
            if all(d is None for d in deltas):
                break
            if not touched:
                before = [(sum(float(np.sum(self.fields[law.fields[f]], dtype=np.float64)) for f in g),
                           sum(float(np.sum(np.abs(self.fields[law.fields[f]].astype(np.float64)))) for f in g))
                          for g in term["conserves"]]
            touched = True
            for (target, _), d in zip(term["equations"], deltas):
                if d is not None:
                    name = law.fields[target]
                    self.fields[name] = (self.fields[name] + d).astype(F32)
        if before is not None:
            for g, (b, scale) in zip(term["conserves"], before):
                after = sum(float(np.sum(self.fields[law.fields[f]], dtype=np.float64)) for f in g)
                tol = 1e-5 * (scale + 1.0) * math.sqrt(count)
                if abs(after - b) > tol:
                    self.violations.append(("conservation", t))
        if touched:
            for w in term["writes"]:
                d = law.decls[w]
                v = self.fields[d["name"]]
                bad = ~np.isfinite(v) | (v < d["lo"]) | (v > d["hi"])
                if d["clamp"]:
                    self.fields[d["name"]] = np.clip(v, d["lo"], d["hi"]).astype(F32)
                elif np.any(bad):
                    self.violations.append(("not-finite" if np.any(~np.isfinite(v)) else "range", t))
