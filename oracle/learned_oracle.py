"""CPU oracle (numpy) of the learned FGMRES preconditioner stage: forward, loss and gradients.

Test infrastructure only: the tests compare the device kernels'
(tubularflowiga_b200/csrc/learned.cu) forward outputs, losses and parameter
gradients with these functions on small meshes.  Nothing in the product path
imports this module.

The network (the definition the kernels implement):
  input    x[node, c]  (4 fields per mesh node, already scaled)
  gather   X[e, 4a + c] = x[conn[e, a], c]  (zero for padded a)          E x 256
  encode   z0 = X Win^T + bin,  h0 = act(z0)                             E x H
  layer l  m_l[e] = mean over the face neighbours e' of h_l[e']  (0 if none)
           z_l = h_l Ws_l^T + m_l Wn_l^T + b_l,  h_{l+1} = h_l + act(z_l)
  decode   y = h_L Wout^T + bout                                         E x 256
  scatter  o[node, c] = s_out[c] / deg(node) * sum_{(e, a): conn[e, a] = node} y[e, 4a + c]
  act(v) = v if v > 0 else 0.1 v
  loss     L = sum_{node, c} w[c] (o[node, c] - t[node, c])^2 / (4 * nodes)
Parameters are one flat FP32 vector: Win (H x 256), bin (H), then per layer
Ws (H x H), Wn (H x H), b (H), then Wout (256 x H), bout (256).
"""
from __future__ import annotations

import numpy as np

SLOPE = 0.1


def act(v):
    return np.where(v > 0, v, SLOPE * v)


def dact(v):
    return np.where(v > 0, 1.0, SLOPE)


def layout(hidden: int, layers: int):
    """Offsets of the parameter blocks in the flat vector."""
    H = hidden
    off = {}
    pos = 0

    def take(name, size):
        nonlocal pos
        off[name] = (pos, size)
        pos += size

    take("Win", H * 256)
    take("bin", H)
    for l in range(layers):
        take(f"Ws{l}", H * H)
        take(f"Wn{l}", H * H)
        take(f"b{l}", H)
    take("Wout", 256 * H)
    take("bout", 256)
    return off, pos


def unpack(theta, hidden, layers):
    off, _ = layout(hidden, layers)
    H = hidden
    p = {}
    for k, (o, s) in off.items():
        v = np.asarray(theta[o:o + s], dtype=np.float64)
        if k == "Win":
            v = v.reshape(H, 256)
        elif k.startswith("Ws") or k.startswith("Wn"):
            v = v.reshape(H, H)
        elif k == "Wout":
            v = v.reshape(256, H)
        p[k] = v
    return p


def pack(grads, hidden, layers):
    off, total = layout(hidden, layers)
    out = np.zeros(total)
    for k, (o, s) in off.items():
        out[o:o + s] = np.ravel(grads[k])
    return out


class Graph:
    def __init__(self, conn, neighbours, nodes):
        self.conn = np.asarray(conn, np.int64)          # E x 64, -1 = padded
        self.nb = np.asarray(neighbours, np.int64)      # E x 6, -1 = none
        self.nodes = nodes
        deg = np.zeros(nodes)
        valid = self.conn >= 0
        np.add.at(deg, self.conn[valid], 1.0)
        self.deg = deg


def forward(theta, graph: Graph, x, s_out, hidden=64, layers=3):
    p = unpack(theta, hidden, layers)
    E = graph.conn.shape[0]
    X = np.zeros((E, 64, 4))
    valid = graph.conn >= 0
    X[valid] = x[graph.conn[valid]]
    X = X.reshape(E, 256)
    cache = {"X": X}
    z0 = X @ p["Win"].T + p["bin"]
    h = act(z0)
    cache["z0"] = z0
    hs, ms, zs = [h], [], []
    nbv = graph.nb >= 0
    cnt = nbv.sum(1)
    for l in range(layers):
        m = np.zeros_like(h)
        for k in range(graph.nb.shape[1]):
            sel = nbv[:, k]
            m[sel] += h[graph.nb[sel, k]]
        m[cnt > 0] /= cnt[cnt > 0, None]
        z = h @ p[f"Ws{l}"].T + m @ p[f"Wn{l}"].T + p[f"b{l}"]
        h = h + act(z)
        ms.append(m)
        zs.append(z)
        hs.append(h)
    y = h @ p["Wout"].T + p["bout"]
    cache.update(hs=hs, ms=ms, zs=zs, y=y, cnt=cnt)
    o = np.zeros((graph.nodes, 4))
    Y = y.reshape(E, 64, 4)
    np.add.at(o, graph.conn[valid], Y[valid])
    o = o * (np.asarray(s_out)[None, :] / np.maximum(graph.deg, 1.0)[:, None])
    return o, cache


def loss(o, t, w):
    d = o - t
    return float(np.sum(np.asarray(w)[None, :] * d * d) / d.size)


def backward(theta, graph: Graph, cache, o, t, w, s_out, hidden=64, layers=3):
    """Gradient of `loss` with respect to the flat parameter vector."""
    p = unpack(theta, hidden, layers)
    E = graph.conn.shape[0]
    do = 2.0 * np.asarray(w)[None, :] * (o - t) / o.size
    do = do * (np.asarray(s_out)[None, :] / np.maximum(graph.deg, 1.0)[:, None])
    valid = graph.conn >= 0
    dY = np.zeros((E, 64, 4))
    dY[valid] = do[graph.conn[valid]]
    dy = dY.reshape(E, 256)
    g = {}
    hs, ms, zs = cache["hs"], cache["ms"], cache["zs"]
    g["Wout"] = dy.T @ hs[-1]
    g["bout"] = dy.sum(0)
    dh = dy @ p["Wout"]
    nbv = graph.nb >= 0
    cnt = cache["cnt"]
    for l in reversed(range(layers)):
        dz = dh * dact(zs[l])
        g[f"Ws{l}"] = dz.T @ hs[l]
        g[f"Wn{l}"] = dz.T @ ms[l]
        g[f"b{l}"] = dz.sum(0)
        dm = dz @ p[f"Wn{l}"]
        dm_scaled = np.zeros_like(dm)
        dm_scaled[cnt > 0] = dm[cnt > 0] / cnt[cnt > 0, None]
        dprev = dh + dz @ p[f"Ws{l}"]
        for k in range(graph.nb.shape[1]):
            sel = nbv[:, k]
            np.add.at(dprev, graph.nb[sel, k], dm_scaled[sel])
        dh = dprev
    dz0 = dh * dact(cache["z0"])
    g["Win"] = dz0.T @ cache["X"]
    g["bin"] = dz0.sum(0)
    return pack(g, hidden, layers)


def face_neighbours(bezier_points, tol=1e-12):
    """Face-adjacent elements from the Bezier nets: two elements share a face when
    the four corner points of one face of each coincide (to `tol` relative to the
    mesh size).  bezier_points: E x 64 x 3, index i + 4 j + 16 k."""
    P = np.asarray(bezier_points).reshape(-1, 64, 3)
    E = P.shape[0]
    scale = np.abs(P).max() if P.size else 1.0
    q = max(tol * scale, 1e-300)
    faces = [(0, 0), (0, 3), (1, 0), (1, 3), (2, 0), (2, 3)]

    def corner(i, j, k):
        return i + 4 * j + 16 * k

    keys = {}
    nb = -np.ones((E, 6), np.int64)
    for e in range(E):
        for f, (axis, side) in enumerate(faces):
            idx = []
            for u in (0, 3):
                for v in (0, 3):
                    ijk = [0, 0, 0]
                    ijk[axis] = side
                    others = [a for a in range(3) if a != axis]
                    ijk[others[0]] = u
                    ijk[others[1]] = v
                    idx.append(corner(*ijk))
            pts = np.round(P[e, idx] / q).astype(np.int64)
            key = tuple(sorted(map(tuple, pts)))
            if key in keys:
                e2, f2 = keys.pop(key)
                nb[e, f] = e2
                nb[e2, f2] = e
            else:
                keys[key] = (e, f)
    return nb
