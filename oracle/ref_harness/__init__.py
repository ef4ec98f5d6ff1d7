"""Harness that runs the reference's own `integrate` kernel — TEST INFRASTRUCTURE ONLY."""
