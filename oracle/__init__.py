"""Oracle package: test infrastructure that checks the device path.

Never imported by the product (maul3d_b200/); see ref.py.
"""
