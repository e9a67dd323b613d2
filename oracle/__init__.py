"""
Oracle for the kinematic-diffraction hot path: test infrastructure, not product.

``oracle.diffraction_oracle`` restates the reference's NumPy ``diffraction()``
(src/python/diffraction.py:62-113).  Only the tests, the smoke check and the
bench's CPU-baseline legs use it, as the checker and as the timed CPU baseline.
"""
