"""Host-side logic of the recorded step (no GPU): the device-decided list mode, the
multi-field stage update's argument checks and the true-entry count of a list."""
import pytest
import torch

from warpsph_b200 import ops
from warpsph_b200.core import AdjacencyList


def test_device_decided_lists_nest_and_suspend():
    assert ops._DEVICE_LISTS[0] == 0
    with ops.device_decided_lists():
        assert ops._DEVICE_LISTS[0] == 1
        with ops.device_decided_lists():
            assert ops._DEVICE_LISTS[0] == 2
            with ops._suspend_device_lists():
                assert ops._DEVICE_LISTS[0] == 0
            assert ops._DEVICE_LISTS[0] == 2
        assert ops._DEVICE_LISTS[0] == 1
    assert ops._DEVICE_LISTS[0] == 0


def test_device_decided_lists_unwind_on_error():
    with pytest.raises(KeyError):
        with ops.device_decided_lists():
            raise KeyError("x")
    assert ops._DEVICE_LISTS[0] == 0


def test_rk_combine_fields_checks_arguments():
    y = torch.zeros(4)
    with pytest.raises(ValueError, match="at most 4"):
        ops.rk_combine_fields(None, [(y, [y], 0)] * 5, [1.0], 1e-3)
    assert ops.rk_combine_fields(None, [], [1.0], 1e-3) == []
    # host tensors never reach a CPU path: the library works on CUDA tensors only
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        ops.rk_combine_fields(None, [(y, [y], 0)], [1.0], 1e-3)


def test_list_entries_of_an_ordinary_list_is_its_nnz():
    offs = torch.tensor([0, 2, 3], dtype=torch.int32)
    cnt = torch.tensor([2, 1, 2], dtype=torch.int32)
    lst = torch.tensor([1, 2, 0, 0, 1], dtype=torch.int32)
    adj = AdjacencyList(neighborOffsets=offs, numNeighbors=cnt, neighborList=lst, numRows=3, numCols=3, nnz=5)
    assert not adj._device_rows
    assert ops.list_entries(adj) == 5
    # a device-decided list reports its capacity as nnz; the true count is read from its rows
    adj_dev = AdjacencyList(neighborOffsets=offs, numNeighbors=cnt, neighborList=torch.zeros(16, dtype=torch.int32), numRows=3,
                            numCols=3, nnz=16)
    adj_dev._device_rows = True
    assert ops.list_entries(adj_dev) == 5
