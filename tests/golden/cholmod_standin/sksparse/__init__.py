"""Test-only stand-in for scikit-sparse (absent from this image).

Only ``sksparse.cholmod`` is provided; see that module.
"""
