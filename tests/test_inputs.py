import numpy as np

from lica_boiling1d_b200.inputs import bubble_poisson_case, face_beta


def test_bubble_case_is_seeded_and_shaped():
    a = bubble_poisson_case(128)
    b = bubble_poisson_case(128)
    np.testing.assert_array_equal(a.rho, b.rho)
    np.testing.assert_array_equal(a.f, b.f)
    assert a.bx.shape == (128, 128) and a.by.shape == (129, 128)
    assert abs(a.f.mean()) < 1e-12
    assert set(np.unique(a.rho)) == {1.0, 1000.0}


def test_face_beta_is_inverse_mean_density():
    rho = np.array([[1.0, 1000.0], [1.0, 1.0]])
    bx, by = face_beta(rho)
    assert bx[0, 1] == 2.0 / 1001.0 and bx[0, 0] == 2.0 / 1001.0
    assert by[1, 1] == 2.0 / 1001.0 and by[2, 0] == 1.0
