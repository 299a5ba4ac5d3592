"""Export and import of simulation systems with the reference's file layout.

Follows src/warpSPH/io.py: exportSimulationSystem (:63-128) writes one file per tag under
``{exportPath}/trajectory/`` with the groups ``adjacency`` (dumpAdjacency, :8-20),
``state`` (dumpState, :22-33) and ``stages/stage_k`` (dumpStage, :35-58: the stage's
update tensors, and under ``aux`` its adjacency and state as ``{k}_adjacency`` and
``{k}_state``), root attributes ``scheme`` and ``time``, and the extra data (tensors as
root datasets, scalars as root attributes, dicts and lists as ``dict_{key}`` groups with
the root attribute set to 'dict' / 'list').  importSimulationSystem (:208-284) reads it
back.  prepExport / importConfigs (:286-316) write and read the run's config.json.

The reference writes HDF5 through h5py.  When h5py is importable the same layout is
written as HDF5 (``{tag}.h5``); otherwise it goes to a numpy archive (``{tag}.npz``) whose
keys are the HDF5 paths (``state/positions``, ``stages/stage_0/aux/1_state/velocities``)
and whose ``__attrs__`` entry holds every group's attributes as JSON.  Tensors keep their
dtypes either way.

Besides the reference's datasets, the adjacency group carries this library's own list
state (``neighborList``, ``interCounts``, and the positions and supports the Verlet rows
were built from), so that an imported system continues with the same Verlet rows -- and
therefore bit for bit -- as the run that exported it.  The reference's loader ignores
datasets it does not name.
"""
from __future__ import annotations

import json
import os
from typing import Any, Optional

import numpy as np
import torch

from . import ops
from .core import AdjacencyList
from .enumTypes import CompressibleSPHScheme, IncompressibleSPHScheme, WeaklyCompressibleSPHScheme
from .integrators import StageRecord

try:  # pragma: no cover - h5py is not part of this image
    import h5py  # type: ignore
except ImportError:  # the numpy-archive form of the same layout
    h5py = None

_NONE = "None"


# ------------------------------------------------------------------ a minimal group tree
class _Group:
    """An in-memory HDF5-like group: datasets (numpy arrays), attributes and subgroups."""

    def __init__(self):
        self.datasets: dict = {}
        self.attrs: dict = {}
        self.groups: dict = {}

    def create_group(self, name: str) -> "_Group":
        g = _Group()
        self.groups[name] = g
        return g

    def create_dataset(self, name: str, data) -> None:
        self.datasets[name] = np.asarray(data)

    def __contains__(self, name: str) -> bool:
        return name in self.groups or name in self.datasets

    def __getitem__(self, name: str):
        return self.groups[name] if name in self.groups else self.datasets[name]


def _json_attr(v):
    if isinstance(v, (np.generic,)):
        return v.item()
    if isinstance(v, torch.Tensor):
        return v.item() if v.numel() == 1 else v.tolist()
    if isinstance(v, (list, tuple)):
        return [_json_attr(x) for x in v]
    return v


def _flatten(g: _Group, prefix: str, arrays: dict, attrs: dict) -> None:
    if g.attrs:
        attrs[prefix] = {k: _json_attr(v) for k, v in g.attrs.items()}
    for k, v in g.datasets.items():
        arrays[f"{prefix}{k}"] = v
    for k, sub in g.groups.items():
        attrs.setdefault(f"{prefix}{k}/", {})
        _flatten(sub, f"{prefix}{k}/", arrays, attrs)


def _unflatten(arrays: dict, attrs: dict) -> _Group:
    root = _Group()

    def group(path: str) -> _Group:
        g = root
        for part in [p for p in path.split("/") if p]:
            g = g.groups.setdefault(part, _Group())
        return g

    for path, a in attrs.items():
        group(path).attrs.update(a)
    for key, v in arrays.items():
        head, _, name = key.rpartition("/")
        group(head).datasets[name] = v
    return root


def _write(tree: _Group, path_no_ext: str) -> str:
    if h5py is not None:  # pragma: no cover
        path = path_no_ext + ".h5"
        with h5py.File(path, "w") as f:
            def put(src: _Group, dst):
                for k, v in src.attrs.items():
                    dst.attrs[k] = v
                for k, v in src.datasets.items():
                    dst.create_dataset(k, data=v)
                for k, sub in src.groups.items():
                    put(sub, dst.create_group(k))
            put(tree, f)
        return path
    path = path_no_ext + ".npz"
    arrays, attrs = {}, {}
    _flatten(tree, "", arrays, attrs)
    arrays["__attrs__"] = np.array(json.dumps(attrs))
    np.savez(path, **arrays)
    return path


def _read(path: str) -> _Group:
    if path.endswith(".h5"):
        if h5py is None:
            raise RuntimeError(f"{path} is an HDF5 file and h5py is not installed")
        with h5py.File(path, "r") as f:  # pragma: no cover
            def get(src) -> _Group:
                g = _Group()
                g.attrs.update(dict(src.attrs))
                for k, v in src.items():
                    if isinstance(v, h5py.Dataset):
                        g.datasets[k] = v[()]
                    else:
                        g.groups[k] = get(v)
                return g
            return get(f)
    with np.load(path, allow_pickle=False) as z:
        arrays = {k: z[k] for k in z.files if k != "__attrs__"}
        attrs = json.loads(str(z["__attrs__"])) if "__attrs__" in z.files else {}
    return _unflatten(arrays, attrs)


def _np(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()


def _torch(a, device) -> torch.Tensor:
    a = np.asarray(a)
    return torch.from_numpy(a.copy()).to(device) if a.shape else torch.tensor(a[()], device=device)


# ------------------------------------------------------------------ dump (io.py:8-58)
def dumpAdjacency(adjacency: AdjacencyList, adjacencyGroup) -> None:
    """io.py:8-20, plus this library's list state (module docstring)."""
    adjacencyGroup.create_dataset("i", data=_np(adjacency.i))
    adjacencyGroup.create_dataset("j", data=_np(adjacency.j))
    adjacencyGroup.create_dataset("numNeighbors", data=_np(adjacency.numNeighbors))
    adjacencyGroup.create_dataset("edgeOffsets", data=_np(adjacency.edgeOffsets))
    for name in ("queryPositions", "querySupports", "referencePositions", "referenceSupports"):
        v = getattr(adjacency, name)
        if v is not None:
            adjacencyGroup.create_dataset(name, data=_np(v))
    adjacencyGroup.attrs["numRows"] = int(adjacency.numRows)
    adjacencyGroup.attrs["numCols"] = int(adjacency.numCols)
    # the library's own list state.  A kept list whose rows are still to be rewritten for
    # its current positions (done on first use) is stored as it stands, with the
    # parameters of that rewrite, so that the imported list is rewritten at the same point
    # of the next step as the exported one would have been
    adjacencyGroup.create_dataset("neighborList", data=_np(adjacency.neighborList))
    if adjacency._pending is not None:
        adjacencyGroup.create_dataset("pendingParams", data=np.frombuffer(bytes(adjacency._pending), dtype=np.uint8))
    elif adjacency.interCounts is not None:
        adjacencyGroup.create_dataset("interCounts", data=_np(adjacency.interCounts))
    if adjacency._x0 is not None:
        adjacencyGroup.create_dataset("buildPositions", data=_np(adjacency._x0))
        adjacencyGroup.create_dataset("buildSupports", data=_np(adjacency._h0))
    adjacencyGroup.attrs["verletScale"] = float(adjacency.verletScale)
    adjacencyGroup.attrs["dim"] = int(adjacency._dim)


_PAIR_FIELDS = ("ap_ij", "av_ij")


def dumpState(state, stateGroup, adjacency: Optional[AdjacencyList] = None) -> None:
    """io.py:22-33: tensors as datasets, None as the attribute 'None', other values as
    attributes.  Pairwise arrays that the step wrote over the interacting prefixes of
    ``adjacency``'s rows are written in the reference's layout (zeros past them)."""
    for fieldName in state.__dict__.keys():
        if fieldName.startswith("_"):
            continue
        fieldValue = getattr(state, fieldName)
        if fieldName in _PAIR_FIELDS and isinstance(fieldValue, torch.Tensor) and adjacency is not None and \
                fieldValue.shape[0] == adjacency.nnz:
            fieldValue, = ops.pair_reference_layout(adjacency, fieldValue)
        if isinstance(fieldValue, torch.Tensor):
            stateGroup.create_dataset(fieldName, data=_np(fieldValue))
        elif fieldValue is None:
            stateGroup.attrs[fieldName] = _NONE
        else:
            stateGroup.attrs[fieldName] = fieldValue


def dumpStage(stage, stageGroups, index: int, SimulationState, exportStagesAdjacency: bool) -> None:
    """io.py:35-58."""
    stageGroups[index].attrs["index"] = index
    auxGroup = stageGroups[index].create_group("aux")
    stageAdjacency = next((a for a in stage.aux if isinstance(a, AdjacencyList)), None)
    for auxIndex, aux in enumerate(stage.aux):
        if isinstance(aux, AdjacencyList):
            if exportStagesAdjacency:
                dumpAdjacency(aux, auxGroup.create_group(f"{auxIndex}_adjacency"))
        elif isinstance(aux, SimulationState):
            dumpState(aux, auxGroup.create_group(f"{auxIndex}_state"), stageAdjacency)
        else:
            print(f"Unsupported aux type: {type(aux)}")
    for updateKey, updateValue in stage.update.__dict__.items():
        if isinstance(updateValue, torch.Tensor):
            stageGroups[index].create_dataset(updateKey, data=_np(updateValue))


def _scheme_name(scheme) -> str:
    return scheme.name if isinstance(scheme, (CompressibleSPHScheme, WeaklyCompressibleSPHScheme, IncompressibleSPHScheme)) else str(scheme)


def exportSimulationSystem(exportPath, tag, scheme, system: Any, exportAdjacency: bool = False, stages=None,
                           exportStagesAdjacency: bool = True, extraData: Optional[dict] = None) -> str:
    """io.py:63-128.  Returns the path written.  As in the reference the system's
    adjacency is written whenever it exists (exportAdjacency is accepted and unused)."""
    outFolderPath = f"{exportPath}/trajectory/"
    os.makedirs(outFolderPath, exist_ok=True)
    out = _Group()
    out.attrs["scheme"] = _scheme_name(scheme)
    out.attrs["time"] = system.t if isinstance(system.t, float) else float(system.t)
    if system.adjacency is not None:
        dumpAdjacency(system.adjacency, out.create_group("adjacency"))
    dumpState(system.state, out.create_group("state"), system.adjacency)
    if stages is not None:
        stageGroups = out.create_group("stages")
        groups = []
        for stageIndex, stage in enumerate(stages):
            groups.append(stageGroups.create_group(f"stage_{stageIndex}"))
            dumpStage(stage, groups, stageIndex, type(system.state), exportStagesAdjacency)
    for key, value in (extraData or {}).items():
        if isinstance(value, dict):
            g = out.create_group(f"dict_{key}")
            for subKey, subValue in value.items():
                if isinstance(subValue, torch.Tensor):
                    g.create_dataset(subKey, data=_np(subValue))
                else:
                    g.attrs[subKey] = subValue
            out.attrs[key] = "dict"
        elif isinstance(value, list):
            g = out.create_group(f"dict_{key}")
            for subIndex, subValue in enumerate(value):
                if isinstance(subValue, torch.Tensor):
                    g.create_dataset(f"{subIndex}", data=_np(subValue))
                elif isinstance(subValue, dict):
                    sg = g.create_group(f"{subIndex}")
                    for k2, v2 in subValue.items():
                        if isinstance(v2, torch.Tensor):
                            sg.create_dataset(k2, data=_np(v2))
                        else:
                            sg.attrs[k2] = v2
                else:
                    g.attrs[f"{subIndex}"] = subValue
            out.attrs[key] = "list"
        elif isinstance(value, torch.Tensor):
            out.create_dataset(key, data=_np(value))
        else:
            out.attrs[key] = value
    return _write(out, f"{outFolderPath}{tag}")


# ------------------------------------------------------------------ load (io.py:146-284)
def loadAdjacency(adjacencyGroup, device) -> AdjacencyList:
    """io.py:146-161.  With the library's list state present the Verlet rows are restored
    as they were exported (interacting prefixes and build state included)."""
    g = adjacencyGroup
    numNeighbors = _torch(g["numNeighbors"], device).to(torch.int32)
    edgeOffsets = _torch(g["edgeOffsets"], device).to(torch.int32)
    lst = _torch(g["neighborList"] if "neighborList" in g else g["j"], device).to(torch.int32)
    qp = _torch(g["queryPositions"], device) if "queryPositions" in g else None
    qs = _torch(g["querySupports"], device) if "querySupports" in g else None
    adj = AdjacencyList(neighborOffsets=edgeOffsets, numNeighbors=numNeighbors, neighborList=lst, numRows=int(g.attrs["numRows"]),
                        numCols=int(g.attrs["numCols"]), nnz=int(lst.shape[0]), queryPositions=qp, querySupports=qs,
                        verletScale=float(g.attrs.get("verletScale", 1.0)))
    if "interCounts" in g:
        adj.interCounts = _torch(g["interCounts"], device).to(torch.int32)
        adj.interNnz = int(adj.interCounts.sum())
    if "pendingParams" in g:
        from . import _capi
        adj._pending = _capi.SphParams.from_buffer_copy(np.ascontiguousarray(g["pendingParams"], dtype=np.uint8).tobytes())
    if "buildPositions" in g:
        adj._x0 = _torch(g["buildPositions"], device)
        adj._h0 = _torch(g["buildSupports"], device)
        adj._dim = int(g.attrs.get("dim", adj._x0.shape[1]))
    return adj


def loadState(stateGroup, device, SimulationState):
    """io.py:163-171: datasets as tensors, attributes as values ('None' back to None)."""
    stateDict = {}
    for k, v in stateGroup.datasets.items():
        stateDict[k] = _torch(v, device)
    for k, v in stateGroup.attrs.items():
        stateDict[k] = None if (isinstance(v, str) and v == _NONE) else v
    return SimulationState(**stateDict)


def loadStage(stageGroup, device, SimulationState, SimulationUpdate) -> StageRecord:
    """io.py:173-190: the aux adjacency and state in index order, and the update."""
    aux = []
    auxGroup = stageGroup["aux"]
    for auxKey in sorted(auxGroup.groups, key=lambda k: int(k.split("_")[0])):
        if auxKey.endswith("_adjacency"):
            aux.append(loadAdjacency(auxGroup.groups[auxKey], device))
        elif auxKey.endswith("_state"):
            aux.append(loadState(auxGroup.groups[auxKey], device, SimulationState))
        else:
            print(f"Unsupported aux type for key {auxKey}")
    updateDict = {k: _torch(v, device) for k, v in stageGroup.datasets.items()}
    return StageRecord(aux=tuple(aux), update=SimulationUpdate(**updateDict))


def schemeNameToSimulationScheme(name: str):
    """io.py:193-201 (incompressible schemes included)."""
    for enum in (CompressibleSPHScheme, WeaklyCompressibleSPHScheme, IncompressibleSPHScheme):
        for scheme in enum:
            if scheme.name.lower() == name.lower():
                return scheme
    raise ValueError(f"Unsupported scheme name: {name}")


def importSimulationSystem(importPath, device, dtype=None, SimulationSystem=None, SimulationState=None, SimulationUpdate=None):
    """io.py:206-284.  Returns (system, stages, scheme, extraData)."""
    f = _read(str(importPath))
    t = f.attrs["time"]
    schemeEnum = schemeNameToSimulationScheme(f.attrs["scheme"])
    if SimulationSystem is None or SimulationState is None or SimulationUpdate is None:
        from .schemes import buildScheme
        SimulationSystem, SimulationState, _, SimulationUpdate, *_ = buildScheme(schemeEnum)
    adjacency = loadAdjacency(f.groups["adjacency"], device) if "adjacency" in f.groups else None
    state = loadState(f.groups["state"], device, SimulationState)
    stages = []
    if "stages" in f.groups:
        sg = f.groups["stages"]
        for stageKey in sorted(sg.groups, key=lambda k: int(k.split("_")[1])):
            stages.append(loadStage(sg.groups[stageKey], device, SimulationState, SimulationUpdate))
    extraData: dict = {}
    for key, value in f.datasets.items():
        extraData[key] = _torch(value, device)
    for key, value in f.attrs.items():
        if key in ("scheme", "time"):
            continue
        if isinstance(value, str) and value in ("dict", "list"):
            g = f.groups[f"dict_{key}"]
            if value == "dict":
                d = {k: _torch(v, device) for k, v in g.datasets.items()}
                d.update(g.attrs)
                extraData[key] = d
            else:
                items = {}
                for k, v in g.datasets.items():
                    items[int(k)] = _torch(v, device)
                for k, sub in g.groups.items():
                    d = {k2: _torch(v2, device) for k2, v2 in sub.datasets.items()}
                    d.update(sub.attrs)
                    items[int(k)] = d
                for k, v in g.attrs.items():
                    items[int(k)] = v
                extraData[key] = [items[k] for k in sorted(items)]
        else:
            extraData[key] = value
    system = SimulationSystem(state=state, adjacency=adjacency, t=t)
    return system, stages, schemeEnum, extraData


# ------------------------------------------------------------------ configs (io.py:286-316)
def prepExport(caseName, config, schemeConfig, scheme, export_fn, exportRoot: str = "export") -> str:
    """io.py:286-308: writes {exportRoot}/{caseName}/config.json with the scheme name,
    the simulation and scheme configurations and a timestamp; returns the export path.
    (The reference fixes exportRoot to 'export', io.py:299-302.)"""
    import datetime
    from .configurations import configurationToDict
    exportPath = f"{exportRoot}/{caseName}"
    os.makedirs(exportPath, exist_ok=True)
    exportDict = {"scheme": _scheme_name(scheme), "config": configurationToDict(config), "schemeConfig": export_fn(schemeConfig),
                  "timestamp": datetime.datetime.now().strftime("%Y-%m-%d_%H-%M-%S")}
    with open(f"{exportPath}/config.json", "w") as fh:
        json.dump(exportDict, fh, indent=4, default=str)
    return exportPath


def importConfigs(configPath, import_fn):
    """io.py:310-316: (SimulationConfig, scheme config) from a config.json."""
    from .configurations import dictToConfig
    with open(configPath, "r") as fh:
        configDict = json.load(fh)
    return dictToConfig(configDict["config"]), import_fn(configDict["schemeConfig"])
