"""Argument checks of the batched product (host side, no GPU needed)."""

import pytest

torch = pytest.importorskip("torch")


def _z(*shape):
    return torch.zeros(shape, dtype=torch.complex128)


def test_validate_accepts_consistent_lists_up_to_the_device_check():
    from bempp_cuda.matmat import validate

    with pytest.raises(ValueError, match="CUDA tensor"):
        validate([_z(3, 4), _z(5, 5)], [_z(4, 2), _z(5, 2)], [_z(3, 2), _z(5, 2)])


@pytest.mark.parametrize("mats,xs,ys,msg", [
    ([], [], [], "non-empty"),
    ([_z(3, 4)], [_z(5, 2)], [_z(3, 2)], "do not match"),
    ([_z(3, 4)], [_z(4, 2)], [_z(4, 2)], "do not match"),
    ([_z(3, 4), _z(2, 2)], [_z(4, 2), _z(2, 3)], [_z(3, 2), _z(2, 3)], "same number"),
    ([_z(3, 4)], [_z(4, 0)], [_z(3, 0)], "no right-hand"),
    ([_z(0, 4)], [_z(4, 1)], [_z(0, 1)], "empty"),
    ([torch.zeros((3, 4))], [_z(4, 1)], [_z(3, 1)], "complex128"),
    ([_z(4, 3).t()], [_z(4, 1)], [_z(3, 1)], "unit column stride"),
    ([_z(3)], [_z(3, 1)], [_z(3, 1)], "2-D"),
])
def test_validate_rejects(mats, xs, ys, msg):
    from bempp_cuda.matmat import validate

    with pytest.raises(ValueError, match=msg):
        validate(mats, xs, ys)
