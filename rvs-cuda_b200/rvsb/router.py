"""Serving across GPUs: requests routed to the least-loaded replica.

Every rank (one process per GPU) holds the scene sets resident and runs its
own serving loop (rvsb_server: continuous batching on that GPU).  Rank 0 is
also the front end: each request goes to the replica with the least
outstanding work, where a request's work is estimated as its output pixels
times the input views of its scene set.  The request's output stays on the
replica that rendered it; what travels is a small descriptor one way and a
completion record (status, batch size, timestamps) back, through a key-value
store beside the process group (torch.distributed.TCPStore).  No collective
and no synthesis data are on the per-request path; the process group is
used only to start and stop together.

Protocol (keys of the store):
  req/<r>/<k>   the k-th request routed to rank r (JSON: id, scene, camera
                fields, synthesis parameters)
  nreq/<r>      number of requests routed to rank r (counter)
  done/<r>/<k>  the k-th completion on rank r (JSON: id, status, batch,
                submit/start/done times on rank r's clock)
  ndone/<r>     number of completions on rank r (counter)
  stop          set by the front end once every request is routed

A replica is any object with submit(scene, camera, params) -> local id and
poll() -> [(local id, status, batch, submit_s, start_s, done_s)]:
ServerReplica adapts rvsb.Server (device output buffers are provided per
request by a caller-supplied allocator); the tests use a host stand-in.
"""
import json
import time

from .abi import Camera, SynthParams


def _to_dict(s):
    out = {}
    for f, _ in s._fields_:
        v = getattr(s, f)
        out[f] = list(v) if hasattr(v, "__len__") else v
    return out


def _from_dict(cls, d):
    s = cls()
    for f, _ in cls._fields_:
        v = d[f]
        if isinstance(v, list):
            getattr(s, f)[:] = v
        else:
            setattr(s, f, v)
    return s


def camera_to_dict(c):
    return _to_dict(c)


def camera_from_dict(d):
    return _from_dict(Camera, d)


def params_to_dict(p):
    return _to_dict(p)


def params_from_dict(d):
    return _from_dict(SynthParams, d)


def request_cost(camera, n_views):
    """Estimated work of one request: output pixels times input views."""
    return float(camera.width) * float(camera.height) * float(max(1, n_views))


class Router:
    """The front end (rank 0): routes requests least-loaded and collects
    their completions."""

    def __init__(self, store, world, scene_views):
        """scene_views: number of input views of each scene set (for the
        cost estimate)."""
        self.store = store
        self.world = world
        self.scene_views = list(scene_views)
        self.routed = [0] * world           # requests sent to each rank
        self.collected = [0] * world        # completions read from each rank
        self.outstanding = [0.0] * world    # estimated work in flight per rank
        self.cost = {}                      # request id -> (rank, cost)
        self.results = {}                   # request id -> completion record
        self.next_id = 0

    def submit(self, scene, camera, params):
        """Routes one request; returns (request id, rank)."""
        self.collect()
        c = request_cost(camera, self.scene_views[scene])
        r = min(range(self.world), key=lambda k: (self.outstanding[k], k))
        rid = self.next_id
        self.next_id += 1
        msg = {"id": rid, "scene": int(scene), "camera": camera_to_dict(camera), "params": params_to_dict(params)}
        self.store.set(f"req/{r}/{self.routed[r]}", json.dumps(msg))
        self.routed[r] += 1
        self.store.add(f"nreq/{r}", 1)
        self.outstanding[r] += c
        self.cost[rid] = (r, c)
        return rid, r

    def collect(self):
        """Reads the completions posted since the last call."""
        for r in range(self.world):
            n = self.store.add(f"ndone/{r}", 0)
            while self.collected[r] < n:
                rec = json.loads(self.store.get(f"done/{r}/{self.collected[r]}"))
                self.collected[r] += 1
                rank, c = self.cost.pop(rec["id"])
                self.outstanding[rank] -= c
                rec["rank"] = rank
                self.results[rec["id"]] = rec

    def finish(self, timeout_s=600.0):
        """Tells the replicas that every request is routed and waits for all
        completions.  Returns the completion records by request id."""
        self.store.set("stop", "1")
        deadline = time.monotonic() + timeout_s
        while len(self.results) < self.next_id:
            self.collect()
            if time.monotonic() > deadline:
                raise TimeoutError(f"{self.next_id - len(self.results)} requests did not complete")
            time.sleep(1e-3)
        return self.results


def serve_replica(store, rank, replica, poll_interval_s=2e-5, timeout_s=600.0):
    """The loop of one replica: takes the requests routed to `rank`, submits
    them to `replica`, posts every completion, and returns once the front end
    has stopped routing and everything routed here has completed.  Returns
    the number of requests served."""
    taken = 0
    posted = 0
    local_to_id = {}
    deadline = time.monotonic() + timeout_s
    stopping = False
    while True:
        n = store.add(f"nreq/{rank}", 0)
        while taken < n:
            msg = json.loads(store.get(f"req/{rank}/{taken}"))
            taken += 1
            lid = replica.submit(msg["scene"], camera_from_dict(msg["camera"]), params_from_dict(msg["params"]))
            local_to_id[lid] = msg["id"]
        done = replica.poll()
        for lid, status, batch, t_submit, t_start, t_done in done:
            rec = {"id": local_to_id.pop(lid), "status": int(status), "batch": int(batch),
                   "submit_s": t_submit, "start_s": t_start, "done_s": t_done}
            store.set(f"done/{rank}/{posted}", json.dumps(rec))
            posted += 1
            store.add(f"ndone/{rank}", 1)
        if not stopping:
            stopping = store.check(["stop"])
        if stopping and not local_to_id and store.add(f"nreq/{rank}", 0) == taken:
            return posted
        if time.monotonic() > deadline:
            raise TimeoutError(f"rank {rank}: {len(local_to_id)} requests still in flight")
        if not done:
            time.sleep(poll_interval_s)


class ServerReplica:
    """rvsb.Server as a replica: scene sets added in the front end's order,
    an output buffer set per request from `alloc(camera)` (kept until the
    request completes, then passed to `on_done(local id, buffers)`)."""

    def __init__(self, server, scene_ids, alloc, on_done=None):
        self.server = server
        self.scene_ids = list(scene_ids)
        self.alloc = alloc
        self.on_done = on_done
        self.held = {}

    def submit(self, scene, camera, params):
        bufs = self.alloc(camera)
        lid = self.server.submit(self.scene_ids[scene], camera, params, bufs)
        self.held[lid] = bufs
        return lid

    def poll(self):
        out = self.server.poll()
        for r in out:
            bufs = self.held.pop(r[0])
            if self.on_done is not None:
                self.on_done(r[0], bufs)
        return out


def open_store(rank, world, host="127.0.0.1", port=None, timeout_s=300):
    """The routing store: served by rank 0 on MASTER_PORT + 1 (or `port`)."""
    import datetime
    import os
    import torch.distributed as dist
    if port is None:
        port = int(os.environ.get("MASTER_PORT", "29500")) + 1
    return dist.TCPStore(host, port, world, rank == 0, timeout=datetime.timedelta(seconds=timeout_s))
